#!/usr/bin/env python
"""Benchmark of the implicit quasi-static LPM load step on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--config sc3d|hex2d]

A step is one quasi-static load step (stiffness assembly, Newton iterations with CG solves,
damage/state update) of the workload.  Default workload: the 3D simple-cubic cube of
20 x 20 x 20 mm at particle radius 0.2 mm (127,500 particles, 382,500 DOF), elastic
E = 200 GPa, nu = 0.25, pulled 0.001 mm per step (20-step path; further steps repeat the
increment).  Inputs are synthetic (the reference's lattice generator).  The stiffness matrix
(~0.56 GB in FP64) exceeds the 126 MB L2, so no flush is needed between steps.

Headline `value`: DOF-iterations per second of the FP64 path (sum over CG iterations of the DOF
count, divided by device time), the reference's own precision.  Beside it: load-step solves/s,
p50/p99 load-step latency, the mixed FP32-Krylov/FP64-refinement path with its displacement
error against the FP64 path, the end-to-end rate through the C ABI with host buffers, the HBM
roofline of the CG kernel and the reference's CPU path timed on this host.

With N > 1 (torchrun) every rank solves its own replica (the path does not shard inside one
solve): value is the sum over ranks, time is the max over ranks, scaling "weak".
"""
from __future__ import annotations

import argparse
import importlib
import json
import os
import re
import shutil
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "LPM solves/sec & DOF-iter/s at ≤1e-6 rel err vs FP64; p50/p99 solve latency"
UNIT = "DOF-iter/s"
NEWTON_TOL = 1e-8  # tight enough that FP64 and mixed agree to 1e-6 in displacement


def args_():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="sc3d", choices=["sc3d", "hex2d"])
    ap.add_argument("--size", type=float, default=20.0, help="specimen edge in mm (20 = the headline workload)")
    ap.add_argument("--no-mixed", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched 64-plate damage workload")
    ap.add_argument("--plates", type=int, default=64, help="plates in the batched damage workload")
    ap.add_argument("--batch-lanes", type=int, default=0,
                    help="lanes of the batch and the server (0: the library's default)")
    ap.add_argument("--no-serving", action="store_true", help="skip the serving-stream leg")
    ap.add_argument("--no-tangent", action="store_true", help="skip the FCC J2 tangent-mode leg")
    ap.add_argument("--no-dump", action="store_true", help="skip the per-step dump output leg")
    ap.add_argument("--no-fatigue", action="store_true", help="skip the fatigue (SolverFatigue) leg")
    ap.add_argument("--no-direct", action="store_true", help="skip the direct-solver (SolverMode::PARDISO) leg")
    ap.add_argument("--autotune", action="store_true",
                    help="tune the CG grid of the headline problem after the first warm-up step (lpmgpu_autotune)")
    ap.add_argument("--tangent-steps", type=int, default=50, help="load steps of the FCC bar's 50-step path timed")
    ap.add_argument("--serve-requests", type=int, default=20, help="requests in the serving-stream sample")
    ap.add_argument("--serve-max-particles", type=float, default=5e5,
                    help="upper end of the log-uniform particle count (the stream's range is 5e3-5e5)")
    return ap.parse_args()


def workload_desc(name, size=20.0):
    """The workload's description and load increment, without building it (both arms use it)."""
    if name == "hex2d":
        return (f"hex2d {size:g}x{size:g} mm r=0.1 plane stress, E=69 GPa, 10 x 0.001 mm top-edge tension",
                10, 0.001)
    dstep = 0.001 * size / 20.0
    return (f"sc3d {size:g}x{size:g}x{size:g} mm r=0.2 elastic, E=200 GPa nu=0.25, 20 x {dstep:g} mm top-face tension",
            20, dstep)


def workload_config(name, size, particles, dim):
    """The `config` object of the JSON line: the same keys and values in both arms."""
    return {"workload": workload_desc(name, size)[0], "particles": int(particles), "dof": int(particles * dim),
            "newton_tol": NEWTON_TOL, "cg_test": "||r||^2 <= 1e-12 ||r0||^2 + 1e-12 (reference)",
            "l2": "stiffness larger than L2 (126 MB); no flush" if name == "sc3d" and size >= 16
            else "stiffness may fit in L2 (126 MB); no flush"}


def workload(name, size=20.0):
    cfg = importlib.import_module("lpm-cpp_b200.configs")
    desc, nsteps, dstep = workload_desc(name, size)
    if name == "hex2d":
        c = cfg.hex_plate(size=size, radius=0.1, steps=nsteps, total_disp=dstep * nsteps, tol_iter=NEWTON_TOL)
    else:
        c = cfg.sc_cube(size=size, radius=0.2, steps=nsteps, total_disp=dstep * nsteps, tol_iter=NEWTON_TOL)
    return c, desc


def reference_spec(name, size, nsteps, tol_iter=NEWTON_TOL, loop="step", solve_threads=0, dump_k=()):
    """Spec of the workload for oracle/_ref/lpm_ref written from the workload's definition alone:
    the reference's own generator builds the lattice, and the boundary groups are coordinate
    conditions evaluated by the driver on the reference's particles (those of
    configs.hex_plate / configs.sc_cube: top and bottom rows within 2r of the box faces; in 3D
    the two bottom corners at minimum y and minimum / maximum x).  Nothing of the product is
    loaded to write it."""
    desc, steps_path, dstep = workload_desc(name, size)
    if name == "hex2d":
        r = 0.1
        lines = ["lattice hex2d", f"radius {r!r}", f"box 0.0 {size!r} 0.0 {size!r} 0.0 1.0", "euler 0 0.0 0.0 0.0",
                 "ptype elastic", "plane_stress 1", "E 69000.0", "mu 0.3", "critical_bstrain 1.0",
                 f"group top 1 > {size - 2 * r!r}", f"group bottom 1 < {2 * r!r}",
                 "settype top 1", "settype bottom 2"]
        bcs = [("bottom", "x", 0.0), ("bottom", "y", 0.0), ("top", "y", dstep)]
    else:
        r = 0.2
        lines = ["lattice sc3d", f"radius {r!r}", f"box 0.0 {size!r} 0.0 {size!r} 0.0 {size!r}", "euler 0 0.0 0.0 0.0",
                 "ptype elastic", "plane_stress 0", "E 200000.0", "mu 0.25", "critical_bstrain 1.0",
                 f"group top 2 > {size - 2 * r!r}", f"group bottom 2 < {2 * r!r}",
                 # the generator's first row in y lies in [0, 2r) and its x rows run from 0 to size
                 f"group corner0 2 < {2 * r!r} 0 < {r!r} 1 < {2 * r!r}",
                 f"group corner1 2 < {2 * r!r} 0 > {size - r!r} 1 < {2 * r!r}",
                 "settype top 1", "settype bottom 2"]
        bcs = [("bottom", "z", 0.0), ("corner0", "x", 0.0), ("corner0", "y", 0.0), ("corner1", "y", 0.0),
               ("top", "z", dstep)]
    lines += ["max_iter 30", f"tol_iter {tol_iter!r}", f"loop {loop}", f"steps {nsteps}"]
    if solve_threads:
        lines.append(f"solve_threads {int(solve_threads)}")
    for g, flag, v in bcs:
        lines.append(f"dispbc {g} {flag} {float(v)!r} 0 {nsteps}")
    for k in dump_k:
        lines.append(f"dumpK {int(k)}")
    return "\n".join(lines) + "\n"


def step_of(case, s):
    return case.load_step(s % len(case.steps))


def algorithmic_bytes_per_iter(nnzb, n, dim, s_k, s_v):
    """Bytes one CG iteration must move: the block matrix (values + int32 block column), the
    row pointers and 9 vector passes (read p, write Ap, read Ap, r/w x, r/w r, r/w p)."""
    return nnzb * (dim * dim * s_k + 4) + (n + 1) * 4 + 9 * dim * n * s_v


def measured_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profiled_traffic(kernel_tag):
    """DRAM bytes per CG iteration from the committed ncu summary, if there is one."""
    path = os.path.join(ROOT, "profiles", f"{kernel_tag}.md")
    try:
        with open(path) as f:
            m = re.search(r"traffic_bytes_per_iter:\s*([0-9.eE+]+)", f.read())
        return float(m.group(1)) if m else None
    except OSError:
        return None


class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        if not shutil.which("nvidia-smi"):
            return
        fd, self.path = tempfile.mkstemp(prefix="clk_", suffix=".csv")
        os.close(fd)
        self.fh = open(self.path, "w")
        self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                      "-lms", "200", "-i", str(self.device)], stdout=self.fh,
                                     stderr=subprocess.DEVNULL)

    def stop(self):
        if not self.proc:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.fh.close()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                t = [x.strip() for x in line.split(",")]
                if len(t) < 9:
                    continue
                try:
                    sm.append(float(t[1]))
                    mx.append(float(t[2]))
                except ValueError:
                    continue
                for k, nm in enumerate(names):
                    if t[5 + k].lower() == "active":
                        reasons.add(nm)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def reduce_ranks(pairs, dist, device):
    """[(value, "max"|"sum"), ...] reduced over the ranks of the process group (identity with
    no group).  Timing is the max over ranks, work is the sum."""
    if dist is None:
        return [float(v) for v, _ in pairs]
    import torch
    out = []
    for v, op in pairs:
        t = torch.tensor([float(v)], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
        out.append(float(t.item()))
    return out


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


# ------------------------------------------------------------------------------------ our arm
def run_ours(a):
    import torch
    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    lpm = importlib.import_module("lpm-cpp_b200.lpm")
    case, desc = workload(a.config, a.size)
    W, K = a.warmup, a.steps

    def barrier():
        if dist:
            dist.barrier()

    def allreduce(v, op):
        return reduce_ranks([(v, op)], dist, "cuda")[0]

    prob = lpm.GpuProblem(case.assembly(), undamaged_pt_type=case.undamaged_type, max_iter=case.max_iter,
                          tol_iter=case.tol_iter, precision=lpm.Precision.FP64, device=local)
    sizes = prob.sizes
    n, dim, nnzb = sizes["n"], sizes["dim"], sizes["nnzb"]
    ndof = n * dim
    stream = torch.cuda.ExternalStream(prob.stream_ptr())
    tune = None
    for s in range(W):
        ok, _ = prob.solve_load_step(step_of(case, s))
        assert ok, f"warm-up step {s} did not converge"
        if s == 0 and a.autotune:
            tune = prob.autotune(iterations=50)
    barrier()
    torch.cuda.synchronize()
    c0 = prob.counters()
    clk = ClockSampler(local)
    clk.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    stats = []
    for s in range(W, W + K):
        ok, st = prob.solve_load_step(step_of(case, s))
        assert ok, f"step {s} did not converge"
        stats.append(st)
    e1.record(stream)
    torch.cuda.synchronize()
    clocks = clk.stop()
    ms = e0.elapsed_time(e1)
    c1 = prob.counters()
    barrier()
    xyz_fp64 = prob.state(("xyz",))["xyz"]

    iters = sum(st["cg_iters"] for st in stats)
    ms_max = allreduce(ms, "max")
    dof_iters_total = allreduce(float(ndof * iters), "sum")
    value = dof_iters_total / (ms_max * 1e-3)
    lat = sorted(st["seconds"] * 1e3 for st in stats)
    cg_s = c1["cg_kernel_seconds"] - c0["cg_kernel_seconds"]
    cg_it = c1["cg_iters"] - c0["cg_iters"]
    cg_launch = c1["cg_launches"] - c0["cg_launches"]
    b_iter = algorithmic_bytes_per_iter(nnzb, n, dim, 8, 8)
    peak, peak_kind = measured_peak()
    achieved = b_iter * cg_it / cg_s / 1e9 if cg_s > 0 else 0.0
    tr = profiled_traffic("cg_fp64_sc3d") if a.config == "sc3d" and a.size == 20.0 else None
    roof = {"bound": "hbm", "kernel": "k_cg<double,double,3> (persistent CG)", "achieved": round(achieved, 1),
            "peak": peak, "unit": "GB/s", "frac": round(achieved / peak, 4), "peak_kind": peak_kind,
            "traffic": (tr * cg_it / max(cg_launch, 1)) if tr else None,
            "algorithmic_bytes_per_iter": b_iter, "iters_per_launch": cg_it / max(cg_launch, 1),
            "avg_launch_ms": cg_s / max(cg_launch, 1) * 1e3}

    # end to end through the C ABI with host buffers: pinned group ids in, positions out
    pin_groups = {}
    for g, ids in case.groups.items():
        t = torch.empty(len(ids), dtype=torch.int32, pin_memory=True)
        t.numpy()[:] = ids
        pin_groups[g] = t
    out = torch.empty((n, 3), dtype=torch.float64, pin_memory=True)
    h2d = 0
    steps_e2e = []
    for s in range(W + K, W + 2 * K):
        disp, force = case.steps[s % len(case.steps)]
        st = lpm.LoadStep()
        for g, fl, v in disp:
            st.dispBCs.append(lpm.DispBC(pin_groups[g].numpy(), lpm.LoadMode.Relative, fl, v))
        for g, fx, fy, fz in force:
            st.forceBCs.append(lpm.ForceBC(pin_groups[g].numpy(), lpm.LoadMode.Relative, fx, fy, fz))
        steps_e2e.append(st)
        h2d = sum(len(b.group) * 4 for b in st.dispBCs + st.forceBCs)
    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e2e_iters = 0
    for st in steps_e2e:
        ok, s2 = prob.solve_load_step(st)
        assert ok
        e2e_iters += s2["cg_iters"]
        prob.read_xyz_into(out.numpy())
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    wall_max = allreduce(wall, "max")
    e2e_total = allreduce(float(ndof * e2e_iters), "sum")
    e2e = {"value": e2e_total / wall_max, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": n * 3 * 8,
           "solves_per_s": world * K / wall_max}
    counters_total = c1["kernel_launches"] - c0["kernel_launches"]
    prob.close()

    # mixed precision on the same path, compared with the FP64 positions after the same steps
    mixed = None
    if not a.no_mixed:
        pm = lpm.GpuProblem(case.assembly(), undamaged_pt_type=case.undamaged_type, max_iter=case.max_iter,
                            tol_iter=case.tol_iter, precision=lpm.Precision.MIXED, device=local)
        sm = torch.cuda.ExternalStream(pm.stream_ptr())
        for s in range(W):
            ok, _ = pm.solve_load_step(step_of(case, s))
            assert ok
        barrier()
        torch.cuda.synchronize()
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record(sm)
        mst = []
        for s in range(W, W + K):
            ok, st = pm.solve_load_step(step_of(case, s))
            assert ok
            mst.append(st)
        f1.record(sm)
        torch.cuda.synchronize()
        mms = allreduce(f0.elapsed_time(f1), "max")
        xm = pm.state(("xyz",))["xyz"]
        u64, um = xyz_fp64 - case.xyz, xm - case.xyz
        err = float(np.linalg.norm(um - u64) / np.linalg.norm(u64))
        miters = sum(st["cg_iters"] for st in mst)
        mixed = {"solves_per_s": world * K / (mms * 1e-3), "ms_per_step": mms / K,
                 "dof_iter_per_s": allreduce(float(ndof * miters), "sum") / (mms * 1e-3),
                 "rel_disp_err_vs_fp64": err, "cg_iters_per_step": miters / K,
                 "speedup_vs_fp64": (ms_max / K) / (mms / K)}
        pm.close()

    # the batched, tangent and serving legs are one-GPU workloads: replicas (N > 1) skip them
    single = world == 1
    batched = None
    if single and not a.no_batched:
        barrier()
        batched = batched_leg(lpm, a.plates, local, world, allreduce, a.batch_lanes)
    tangent = None
    if single and not a.no_tangent:
        barrier()
        tangent = tangent_leg(lpm, a.tangent_steps, local, world, allreduce)
    dump = None
    if single and not a.no_dump:
        barrier()
        dump = dump_leg(lpm, case, W, local)
    serving = None
    if single and not a.no_serving:
        barrier()
        serving = serving_leg(lpm, a.serve_requests, a.serve_max_particles, local, world, allreduce, a.batch_lanes)

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        try:
            cpu = cpu_baseline(a.config, a.size)
            if cpu.get("kind") == "reference":
                cpu["parity"] = reference_parity(lpm, local)
        except Exception as ex:  # the baseline must not cost the bench line
            cpu = {"error": f"{type(ex).__name__}: {ex}"}
    # last, after every other measurement: the newest device path
    fatigue = None
    if single and not a.no_fatigue:
        fatigue = fatigue_leg(lpm, local)
    direct = None
    if single and not a.no_direct:
        direct = direct_leg(lpm, local)

    if rank == 0:
        # every leg in full on its own line first; the last line is the compact record
        for name, leg in (("mixed", mixed), ("batched", batched), ("tangent", tangent), ("dump", dump),
                          ("serving", serving), ("cpu_baseline", cpu), ("fatigue", fatigue), ("direct", direct)):
            if leg is not None:
                print(json.dumps({"leg": name, **leg}), flush=True)
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
            "ms_per_step": ms_max / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic (reference lattice generator)",
            "config": workload_config(a.config, a.size, n, dim),
            "roofline": roof, "e2e": e2e, "gpu_launches": counters_total, "clocks": clocks,
            "cpu_baseline": _r({k: v for k, v in (cpu or {}).items() if k != "parity"}) if cpu else None,
            "solves_per_s": world * K / (ms_max * 1e-3),
            "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99))},
            "newton_per_step": sum(st["newton_solves"] for st in stats) / K,
            "cg_iters_per_step": iters / K,
            "phases_ms_per_step": {"assembly": (c1["assembly_seconds"] - c0["assembly_seconds"]) * 1e3 / K,
                                   "force": (c1["force_seconds"] - c0["force_seconds"]) * 1e3 / K,
                                   "cg_kernel": cg_s * 1e3 / K},
            "parallelism": f"replicas x{world}", "cg_grid": tune if tune is not None else "default",
            "sizes": {"block_nnz": nnzb, "nnz_upper_ref_csr": sizes["nnz_upper"]},
            "legs": compact_legs(mixed, batched, serving, tangent, dump, cpu, fatigue, direct),
        }
        print(json.dumps(_r(line), separators=(",", ":")), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def _r(o, sig=4):
    """Floats rounded to `sig` significant digits, recursively (keeps the record short)."""
    if isinstance(o, float):
        return float(f"{o:.{sig}g}") if o == o and abs(o) != float("inf") else o
    if isinstance(o, dict):
        return {k: _r(v, sig) for k, v in o.items()}
    if isinstance(o, (list, tuple)):
        return [_r(v, sig) for v in o]
    return o


def compact_legs(mixed, batched, serving, tangent, dump, cpu, fatigue, direct):
    """The other measurements in a few keys each (the full objects are printed above the line)."""
    out = {}

    def err(leg):
        return {"error": leg["error"][:160]} if isinstance(leg, dict) and "error" in leg else None

    if mixed:
        out["mixed"] = {"speedup_vs_fp64": mixed["speedup_vs_fp64"], "rel_disp_err_vs_fp64": mixed["rel_disp_err_vs_fp64"],
                        "dof_iter_per_s": mixed["dof_iter_per_s"], "ms_per_step": mixed["ms_per_step"]}
    if batched:
        out["batched"] = err(batched) or {
            "specimens": batched.get("specimens"),
            "plain_fp64_solves_per_s": batched["plain_fp64_one_at_a_time"]["solves_per_s"],
            "batched_mixed_solves_per_s": batched["batched_mixed"]["solves_per_s"],
            "speedup_batched_mixed_vs_plain_fp64": batched["speedup_batched_mixed_vs_plain_fp64"],
            "speedup_batched_fp64_vs_plain_fp64": batched["speedup_batched_fp64_vs_plain_fp64"],
            "max_rel_disp_err_mixed_vs_plain_fp64": batched["batched_mixed"]["max_rel_disp_err_vs_plain_fp64"]}
    if serving:
        out["serving"] = err(serving) or {
            "requests": serving.get("requests"), "particles_range": serving.get("particles_range"),
            "plain_fp64_solves_per_s": serving["plain_fp64_one_at_a_time"]["solves_per_s"],
            "served_mixed_solves_per_s": serving["served_mixed"]["solves_per_s"],
            "served_mixed_latency_s": serving["served_mixed"]["latency_s"],
            "plain_fp64_latency_s": serving["plain_fp64_one_at_a_time"]["latency_s"],
            "speedup_served_mixed_vs_plain_fp64": serving["speedup_served_mixed_vs_plain_fp64"],
            "max_rel_disp_err_mixed_vs_plain_fp64": serving["served_mixed"]["max_rel_disp_err_vs_plain_fp64"]}
    if tangent:
        out["tangent"] = err(tangent) or {
            "steps_timed": tangent.get("steps_timed"), "fp64_ms_per_step": tangent["fp64"]["ms_per_step"],
            "mixed_ms_per_step": tangent["mixed"]["ms_per_step"], "speedup_mixed_vs_fp64": tangent["speedup_mixed_vs_fp64"],
            "rel_disp_err_mixed_vs_fp64": tangent["mixed"]["rel_disp_err_vs_fp64"],
            "assembly_share_fp64": tangent["fp64"]["assembly_share"]}
    if cpu and isinstance(cpu.get("parity"), dict):
        p = cpu["parity"]
        out["parity_vs_reference"] = err(p) or {"workload": p.get("workload_short"),
                                                "fp64_rel_disp": p["fp64"]["rel_disp_err_vs_reference"],
                                                "mixed_rel_disp": p["mixed"]["rel_disp_err_vs_reference"]}
    if dump:
        out["dump"] = err(dump) or {"ms_exposed_async": dump.get("dump_ms_exposed_async"),
                                    "ms_sync": dump.get("dump_ms_sync")}
    if fatigue:
        out["fatigue"] = err(fatigue) or {"speedup_vs_reference": fatigue.get("speedup_vs_reference"),
                                          "max_abs_damage_diff": fatigue.get("max_abs_damage_diff_vs_reference")}
    if direct:
        out["direct"] = err(direct) or {k: {"cg_ms": v["cg"]["ms_per_step"], "direct_ms": v["direct"]["ms_per_step"]}
                                        for k, v in direct.items() if isinstance(v, dict) and "cg" in v}
    return out


def dump_leg(lpm, case, first_step, device, steps=3):
    """Per-step output on the headline cube: lpmgpu_dump_write appends each load step's state in
    the reference's dump text (Assembly::writeDump, include/assembly.h:310-335), formatted on all
    host cores.  Three arms of `steps` FP64 load steps each, wall time: the steps alone, each step
    followed by a synchronous dump, and each step's dump written by the writer thread while the
    next step runs (flushed at the end).  Errors are reported in the line, not raised."""
    import shutil
    import tempfile
    import torch
    d = tempfile.mkdtemp(prefix="lpm_dump_")
    try:
        prob = lpm.GpuProblem(case.assembly(), undamaged_pt_type=case.undamaged_type, max_iter=case.max_iter,
                              tol_iter=case.tol_iter, precision=lpm.Precision.FP64, device=device)
        s = first_step
        ok, _ = prob.solve_load_step(step_of(case, s))
        s += 1
        arms = {}
        for arm in ("steps_only", "sync_dump", "async_dump"):
            path = os.path.join(d, arm + ".dump")
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            for _ in range(steps):
                ok, _ = prob.solve_load_step(step_of(case, s))
                if not ok:
                    raise RuntimeError(f"load step {s} did not converge")
                if arm != "steps_only":
                    prob.dump_write(path, s, case.box, threads=0, async_=(arm == "async_dump"))
                s += 1
            prob.dump_flush()
            torch.cuda.synchronize()
            arms[arm] = (time.perf_counter() - t0) * 1e3 / steps
        size = os.path.getsize(os.path.join(d, "sync_dump.dump")) / steps
        prob.close()
        return {"particles": case.n, "bytes_per_step": size, "host_threads": os.cpu_count(),
                "ms_per_step": arms,
                "dump_ms_sync": arms["sync_dump"] - arms["steps_only"],
                "dump_ms_exposed_async": arms["async_dump"] - arms["steps_only"]}
    except Exception as ex:  # the leg must not cost the bench line
        return {"error": f"{type(ex).__name__}: {ex}"}
    finally:
        shutil.rmtree(d, ignore_errors=True)


def direct_leg(lpm, device, sizes=(10.0, 20.0), steps=3):
    """The direct solver (SolverMode::PARDISO's role; lpmgpu_desc.direct = 1) against the CG on
    the hexagonal plate of config 1 (r = 0.1 mm, 10 x 10 mm: 2,900 particles; 20 x 20 mm: 11,500),
    `steps` load steps of 0.001 mm at Newton tolerance 1e-8, the CG at 1e-24 on squared norms.
    Device time of the library's stream per load step; the first step of the direct path includes
    the ordering and the band's allocation.  Error: the direct displacements against the CG's."""
    try:
        import torch
        cfg = importlib.import_module("lpm-cpp_b200.configs")
        out = {}
        for size in sizes:
            c = cfg.hex_plate(size=size, radius=0.1, steps=steps, total_disp=0.001 * steps, tol_iter=NEWTON_TOL)
            row, xyz = {}, {}
            for key, mode in (("cg", 0), ("direct", 1)):
                g = lpm.GpuProblem(c.assembly(), undamaged_pt_type=c.undamaged_type, max_iter=c.max_iter,
                                   tol_iter=c.tol_iter, cg_rtol=1e-24, cg_atol=0.0, device=device, direct=mode)
                s0 = torch.cuda.ExternalStream(g.stream_ptr())
                torch.cuda.synchronize()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(s0)
                newton = 0
                for s in range(steps):
                    ok, st = g.solve_load_step(c.load_step(s))
                    assert ok, f"{key} step {s} failed"
                    newton += st["newton_solves"]
                e1.record(s0)
                torch.cuda.synchronize()
                row[key] = {"ms_per_step": e0.elapsed_time(e1) / steps, "newton_per_step": newton / steps}
                xyz[key] = g.state(("xyz",))["xyz"] - c.xyz
                g.close()
            row["rel_disp_diff_direct_vs_cg"] = float(np.linalg.norm(xyz["direct"] - xyz["cg"]) /
                                                      np.linalg.norm(xyz["cg"]))
            out[f"hex_{size:g}mm_{c.n}"] = row
        return out
    except Exception as ex:  # the leg must not cost the bench line
        return {"error": f"{type(ex).__name__}: {ex}"}


def fatigue_leg(lpm, device, size=25.0, cycles=4):
    """Fatigue (SolverFatigue, include/solver_fatigue.h) on a hexagonal plate of fatigue HCF
    particles (lpm-cpp_b200/configs.fatigue_plate): `size` mm at r = 0.1, nonlocal averaging over
    1.5 x 0.3 mm, one static step of solveProblemStatic, then `cycles` displacement cycles of
    solveProblemCyclic (LoadUniaxialDisp, two steps up and two down, the amplitude scaled to the
    plate so that the strain is that of the 2.4 mm test plate; dN/dt = 2), at the example's Newton
    tolerance 1e-5 and the reference's CG test.  GPU: the C ABI steps, wall time around the
    host-driven calls (creation and the nonlocal search untimed).  Reference: the reference's own
    SolverFatigue (oracle/_ref/lpm_ref) on all host cores, the same spec, wall time of the same
    static step and cycles.  Error: the final damage and displacements against the reference run
    (both stop at the loose tolerance, and the reference's assembly races at several threads)."""
    try:
        import torch
        from oracle import oracle as O
        cfg = importlib.import_module("lpm-cpp_b200.configs")
        c = cfg.fatigue_plate(size=size, radius=0.1, cycles=cycles, amplitude=0.004 * size / 2.4, tol_iter=1e-5)
        fat = c.meta["fatigue"]
        amp = max(abs(v) for v in fat["spectrum"])
        groups = [c.groups[g] for g in fat["groups"]]
        g = lpm.GpuProblem(c.assembly(), undamaged_pt_type=c.undamaged_type, max_iter=c.max_iter,
                           tol_iter=c.tol_iter, device=device)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ok, st = g.fatigue_static_step(c.load_step(0))
        assert ok, "static step did not converge"
        newton, ncyc, N = st["newton_solves"], 0, 0
        n_cycles = 0.5 * (len(fat["spectrum"]) - 1)
        while True:  # solveProblemCyclic's loop (solver_fatigue.h:183-218)
            steps = lpm.generateLoadCycle(lpm.FatigueLoadType.LoadUniaxialDisp, fat["spectrum"], N, fat["n_interval"],
                                          groups)
            dNdt = lpm.func_dNdt_linear(fat["tau"])
            _, st = g.fatigue_cycle(steps, dNdt)
            newton += st["newton_solves"]
            ncyc += 1
            N += dNdt
            if not N < n_cycles:
                break
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
        sg = g.state(("xyz", "damage"))
        g.close()
        out = {"workload": f"fatigue HCF hex plate {size:g} mm, r=0.1 ({c.n} particles), 1 static step + {ncyc} "
                           f"cycles x 4 steps, dN/dt={dNdt}, Newton tol 1e-5",
               "gpu": {"seconds": wall, "cycles_per_s": ncyc / wall, "newton_solves": newton,
                       "max_damage": float(sg["damage"].max())}}
        if O.ref_available():
            threads = os.cpu_count() or 1
            d = tempfile.mkdtemp(prefix="lpmref_fatigue_")
            try:
                O.run_ref(O.write_ref_spec(c, d, loop="ref"), d, threads=threads, timeout=1800)
                rows = O.read_ref_steps(d)
                last = len(rows) - 1
                xr = O.read_bin(d, f"xyz_{last:03d}.f64", np.float64).reshape(-1, 3)
                dr = O.read_bin(d, f"damage_{last:03d}.f64", np.float64)
            finally:
                shutil.rmtree(d, ignore_errors=True)
            wall_r = sum(r["wall_s"] for r in rows)
            # the leg's CPU baseline and checker: the reference's own SolverFatigue on the host cores
            out["cpu_baseline"] = {"seconds": wall_r, "cycles_per_s": ncyc / wall_r, "cores": threads,
                                   "kind": "reference", "newton_solves": int(sum(r["newton_solves"] for r in rows)),
                                   "sample": "the same static step and cycles"}
            out["speedup_vs_reference"] = wall_r / wall
            out["max_abs_damage_diff_vs_reference"] = float(np.abs(sg["damage"] - dr).max())
            out["max_abs_disp_diff_vs_reference_over_amplitude"] = float(np.abs(sg["xyz"] - xr).max() / amp)
        try:
            out["batched"] = fatigue_batch_sample(lpm, device)
        except Exception as ex:  # keeps the single-specimen numbers above
            out["batched"] = {"error": f"{type(ex).__name__}: {ex}"}
        return out
    except Exception as ex:  # the leg must not cost the bench line
        return {"error": f"{type(ex).__name__}: {ex}"}


def fatigue_batch_sample(lpm, device, sizes=(4.0, 5.0, 6.0, 7.0, 8.0, 9.0, 10.0, 12.0)):
    """Eight fatigue plates of uneven size (the 2.4 mm test plate's strain and rate law, one static
    step and two simulated cycles each): one at a time through the C ABI's fatigue steps, then all
    as fatigue members of one batch (lpmgpu_batch_add_fatigue); wall time of each, problem
    creation untimed, and the largest damage difference between the two."""
    import torch
    cfg = importlib.import_module("lpm-cpp_b200.configs")
    cases = [cfg.fatigue_plate(size=sz, radius=0.1, cycles=4, amplitude=0.004 * sz / 2.4, tol_iter=1e-5)
             for sz in sizes]
    cyc = []
    for c in cases:
        fat, N, lst = c.meta["fatigue"], 0, []
        while True:
            steps = lpm.generateLoadCycle(lpm.FatigueLoadType.LoadUniaxialDisp, fat["spectrum"], N, fat["n_interval"],
                                          [c.groups[g] for g in fat["groups"]])
            d = lpm.func_dNdt_linear(fat["tau"])
            lst.append((steps, d))
            N += d
            if not N < 0.5 * (len(fat["spectrum"]) - 1):
                break
        cyc.append(lst)

    def make(c):
        return lpm.GpuProblem(c.assembly(), undamaged_pt_type=c.undamaged_type, max_iter=c.max_iter,
                              tol_iter=c.tol_iter, device=device)
    probs = [make(c) for c in cases]
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for g, c, lst in zip(probs, cases, cyc):
        g.fatigue_static_step(c.load_step(0))
        for steps, d in lst:
            g.fatigue_cycle(steps, d)
    torch.cuda.synchronize()
    t_plain = time.perf_counter() - t0
    dmg_plain = [g.state(("damage",))["damage"] for g in probs]
    for g in probs:
        g.close()
    probs = [make(c) for c in cases]
    b = lpm.Batch(device)
    for g, c, lst in zip(probs, cases, cyc):
        b.add_fatigue(g, [c.load_step(0)], [x[0] for x in lst], [x[1] for x in lst])
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    b.run()
    torch.cuda.synchronize()
    t_batch = time.perf_counter() - t0
    diff = max(float(np.abs(g.state(("damage",))["damage"] - d0).max()) for g, d0 in zip(probs, dmg_plain))
    b.close()
    for g in probs:
        g.close()
    return {"specimens": len(cases), "particles": int(sum(c.n for c in cases)),
            "plain_s": t_plain, "batched_s": t_batch, "speedup_batched_vs_plain": t_plain / t_batch,
            "max_damage_diff_batched_vs_plain": diff}


def batched_leg(lpm, count, device, world, allreduce, lanes=0):
    """Batched 2D damage workload (lpm-cpp_b200/configs.batched_notched_plates): `count` seeded
    single-edge-notched hexagonal plates of uneven size, 40 Mode-I steps each, solved (1) one
    plate at a time on the plain FP64 path, (2) all together by one batch in FP64, (3) all
    together by one batch in mixed precision.  A solve is one plate's whole 40-step path.
    Wall time around the host calls (the batch is host-driven); problem creation is outside
    the timed regions.  Errors: final displacement of each plate against the plain FP64 path."""
    import torch
    cfg = importlib.import_module("lpm-cpp_b200.configs")
    cases = cfg.batched_notched_plates(count=count)

    def make(c, prec):
        return lpm.GpuProblem(c.assembly(), undamaged_pt_type=c.undamaged_type, max_iter=c.max_iter,
                              tol_iter=c.tol_iter, precision=lpm.Precision(prec), device=device)

    # (1) plain FP64, one plate after another
    plain_u, plain_s, plain_di, lat_plain = [], 0.0, 0, []
    for c in cases:
        g = make(c, 0)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        iters = 0
        for s in range(len(c.steps)):
            ok, st = g.solve_load_step(c.load_step(s))
            assert ok, f"{c.name}: step {s} failed on the plain path"
            iters += st["cg_iters"]
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        plain_s += dt
        lat_plain.append(dt)
        plain_di += iters * c.n * 2
        plain_u.append(g.state(("xyz",))["xyz"] - c.xyz)
        g.close()

    def batch_run(prec):
        gs = [make(c, prec) for c in cases]
        b = lpm.Batch(device)
        if lanes > 0:
            b.set_lanes(lanes)
        mids = [b.add(g, [c.load_step(s) for s in range(len(c.steps))]) for g, c in zip(gs, cases)]
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        b.run()
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        st = b.stats()
        errs, lat = [], []
        for g, c, mid, u0 in zip(gs, cases, mids, plain_u):
            info = b.member(mid)
            assert info["state"] == 1, f"{c.name}: {info}"
            lat.append(info["seconds"])
            u = g.state(("xyz",))["xyz"] - c.xyz
            errs.append(float(np.linalg.norm(u - u0) / np.linalg.norm(u0)))
        b.close()
        for g in gs:
            g.close()
        tmax = allreduce(dt, "max")
        return {"seconds": tmax, "solves_per_s": world * count / tmax,
                "dof_iter_per_s": allreduce(float(st["dof_iters"]), "sum") / tmax,
                "rounds": st["rounds"], "cg_launches": st["cg_launches"],
                "cg_kernel_seconds": st["cg_kernel_seconds"],
                "latency_s": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99))},
                "max_rel_disp_err_vs_plain_fp64": max(errs), "median_rel_disp_err_vs_plain_fp64": float(np.median(errs))}

    fp64 = batch_run(0)
    mixed = batch_run(1)
    pmax = allreduce(plain_s, "max")
    plain = {"seconds": pmax, "solves_per_s": world * count / pmax,
             "dof_iter_per_s": allreduce(float(plain_di), "sum") / pmax,
             "latency_s": {"p50": float(np.percentile(lat_plain, 50)), "p99": float(np.percentile(lat_plain, 99))}}
    return {"workload": f"{count} single-edge-notched hex plates, side log-uniform 4-25 mm at r=0.1 mm, "
                        f"slit 0.2-0.5 of width, E 60-120 GPa, critical stretch 1e-3-3e-3, 40 Mode-I steps "
                        f"({sum(c.n for c in cases)} particles, seed {cases[0].meta['seed']})",
            "lanes": lanes if lanes > 0 else "default",
            "plain_fp64_one_at_a_time": plain, "batched_fp64": fp64, "batched_mixed": mixed,
            "speedup_batched_mixed_vs_plain_fp64": mixed["solves_per_s"] / plain["solves_per_s"],
            "speedup_batched_fp64_vs_plain_fp64": fp64["solves_per_s"] / plain["solves_per_s"]}


def tangent_leg(lpm, steps, device, world, allreduce):
    """FCC single-crystal bar in J2 plasticity with the tangent re-assembled before every Newton
    solve (lpm-cpp_b200/configs.fcc_bar): 16 x 16 x 32 mm at r = 0.18 mm (248,319 particles,
    lattice constant 0.509 mm), seeded uniform orientation, E 110 GPa, nu 0.34, sigma_y = CRSS 60 MPa
    x Taylor factor 3.06, H = 500 MPa, tension to 1% strain in 50 steps.  The first `steps` steps
    of the path are timed (a bounded sample), in FP64 and in mixed precision (FP32 Krylov in FP64
    refinement; the return mapping and the assembly stay FP64); device time of the library's
    stream.  Error: the mixed displacement against FP64 after the same steps."""
    import torch
    cfg = importlib.import_module("lpm-cpp_b200.configs")
    c = cfg.fcc_bar(size=(16.0, 16.0, 32.0), radius=0.18, steps=50, strain=0.01)
    out, xyz = {}, {}
    for prec, key in ((0, "fp64"), (1, "mixed")):
        g = lpm.GpuProblem(c.assembly(), undamaged_pt_type=c.undamaged_type, max_iter=c.max_iter,
                           tol_iter=NEWTON_TOL, precision=lpm.Precision(prec), device=device, tangent=True)
        s0 = torch.cuda.ExternalStream(g.stream_ptr())
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        c0 = g.counters()
        e0.record(s0)
        newton = iters = 0
        for s in range(steps):
            ok, st = g.solve_load_step(c.load_step(s))
            assert ok, f"FCC bar step {s} failed"
            newton += st["newton_solves"]
            iters += st["cg_iters"]
        e1.record(s0)
        torch.cuda.synchronize()
        ms = allreduce(e0.elapsed_time(e1), "max")
        c1 = g.counters()
        xyz[key] = g.state(("xyz",))["xyz"]
        out[key] = {"ms_per_step": ms / steps, "dof_iter_per_s": allreduce(float(iters * c.n * 3), "sum") / (ms * 1e-3),
                    "newton_per_step": newton / steps, "cg_iters_per_step": iters / steps,
                    "assembly_ms_per_newton": (c1["assembly_seconds"] - c0["assembly_seconds"]) * 1e3 / max(newton, 1),
                    "assembly_share": (c1["assembly_seconds"] - c0["assembly_seconds"]) / (ms * 1e-3)}
        g.close()
    u64, um = xyz["fp64"] - c.xyz, xyz["mixed"] - c.xyz
    out["mixed"]["rel_disp_err_vs_fp64"] = float(np.linalg.norm(um - u64) / np.linalg.norm(u64))
    out["speedup_mixed_vs_fp64"] = out["fp64"]["ms_per_step"] / out["mixed"]["ms_per_step"]
    out["workload"] = (f"FCC J2 bar 16x16x32 mm, r=0.18 ({c.n} particles), tangent re-assembled every Newton "
                       f"iteration, {'all 50' if steps >= 50 else f'first {steps} of 50'} steps to 1% strain, "
                       f"Newton tol {NEWTON_TOL}")
    out["steps_timed"] = f"{steps}/50"
    return out


def serving_leg(lpm, count, nmax, device, world, allreduce, lanes=0):
    """Serving stream (lpm-cpp_b200/configs.serving_requests): `count` requests with seeded
    Poisson arrivals (mean 200/s) of elastic or J2 solves on hex-2D / SC-3D / BCC-3D lattices,
    particle count log-uniform 5e3..`nmax`, 5-50 monotone steps each.
      plain     the FP64 path one request at a time in arrival order (create + all steps, timed
                per request; each request starts when it has arrived and the previous one is
                done, so its latency includes queueing);
      served    lpm.Server (HBM budget 150 GB, continuous batching), each request submitted at
                its arrival time, in mixed precision and in FP64.
    solves/s = requests / (last completion - first arrival); latency = completion - arrival.
    Errors: each request's final displacement against the plain FP64 result."""
    import threading
    import torch
    cfg = importlib.import_module("lpm-cpp_b200.configs")
    reqs = cfg.serving_requests(count=count, n_range=(5e3, nmax))
    for _, c in reqs:
        # the headline's Newton tolerance, so that mixed and FP64 results stay within 1e-6
        c.tol_iter = NEWTON_TOL
    steps_of = lambda c: [c.load_step(s) for s in range(len(c.steps))]  # noqa: E731

    # plain FP64, one at a time
    clock, lat_plain, u_plain, dof_iters = 0.0, [], [], 0
    for arr, c in reqs:
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        g = lpm.GpuProblem(c.assembly(), undamaged_pt_type=c.undamaged_type, max_iter=c.max_iter,
                           tol_iter=c.tol_iter, device=device)
        for st in steps_of(c):
            ok, s2 = g.solve_load_step(st)
            assert ok, f"{c.name}: plain path failed"
            dof_iters += s2["cg_iters"] * c.n * c.dim
        u_plain.append(g.state(("xyz",))["xyz"] - c.xyz)
        g.close()
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        clock = max(clock, arr) + dt
        lat_plain.append(clock - arr)
    span_plain = clock - reqs[0][0]

    def served(prec):
        srv = lpm.Server(device=device, hbm_budget_bytes=150 * 10**9)
        if lanes > 0:
            srv.set_lanes(lanes)
        ids = [None] * len(reqs)
        t_base = time.perf_counter()

        def submitter():
            for k, (arr, c) in enumerate(reqs):
                wait = arr - (time.perf_counter() - t_base)
                if wait > 0:
                    time.sleep(wait)
                ids[k] = srv.submit(c.assembly(), steps_of(c), undamaged_pt_type=c.undamaged_type,
                                    max_iter=c.max_iter, tol_iter=c.tol_iter, precision=lpm.Precision(prec))

        th = threading.Thread(target=submitter)
        th.start()
        th.join()
        lat, errs, end, first = [], [], 0.0, float("inf")
        for k, (arr, c) in enumerate(reqs):
            info = srv.wait(ids[k], timeout=3600)
            assert info["state"] == 2, f"{c.name}: {info}"
            u = srv.result(ids[k]) - c.xyz
            errs.append(float(np.linalg.norm(u - u_plain[k]) / np.linalg.norm(u_plain[k])))
            # times on the server's clock; arrivals on the submitter's
            lat.append(info["t_done"] - info["t_submit"])
            end = max(end, info["t_done"])
            first = min(first, info["t_submit"])
        st = srv.stats()
        srv.close()
        span = end - first
        return {"solves_per_s": world * len(reqs) / allreduce(span, "max"), "makespan_s": span,
                "latency_s": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99))},
                "rounds": st["rounds"], "peak_device_bytes": st["peak_bytes"],
                "max_rel_disp_err_vs_plain_fp64": max(errs), "median_rel_disp_err_vs_plain_fp64": float(np.median(errs))}

    mixed = served(1)
    fp64 = served(0)
    plain = {"solves_per_s": world * len(reqs) / allreduce(span_plain, "max"), "makespan_s": span_plain,
             "latency_s": {"p50": float(np.percentile(lat_plain, 50)), "p99": float(np.percentile(lat_plain, 99))},
             "dof_iter_per_s": dof_iters / span_plain}
    return {"workload": f"{len(reqs)} requests, Poisson arrivals 200/s (seed {reqs[0][1].meta['seed']}); hex-2D / "
                        f"SC-3D / BCC-3D, N log-uniform 5e3-{nmax:.0e} (the stream's range is 5e3-5e5), "
                        f"E 50-250 GPa, nu 0.2-0.35, Newton tol {NEWTON_TOL}, 5-50 steps to "
                        f"0.1% strain, elastic or J2; {sum(c.n for _, c in reqs)} particles in total",
            "requests": len(reqs), "particles_range": [int(min(c.n for _, c in reqs)), int(max(c.n for _, c in reqs))],
            "plain_fp64_one_at_a_time": plain, "served_mixed": mixed, "served_fp64": fp64,
            "speedup_served_mixed_vs_plain_fp64": mixed["solves_per_s"] / plain["solves_per_s"],
            "hbm_budget_bytes": 150 * 10**9}


# ------------------------------------------------------------------------------------ CPU legs
def reference_parity(lpm, device, size=6.0, steps=3):
    """The errors of the device solutions against the reference's own FP64 solution: the SC cube of
    the headline workload at `size` mm (r = 0.2), `steps` load steps, the bench's Newton tolerance
    and the reference's CG test, solved by oracle/_ref/lpm_ref single-threaded (its multi-threaded
    assembly races) and on the device in FP64 and mixed precision.  Per arm: the largest relative
    displacement error over the steps and the relative error of the reaction-force norm."""
    try:
        from oracle import oracle as O
        case, desc = workload("sc3d", size)
        case.steps = case.steps[:steps]
        d = tempfile.mkdtemp(prefix="lpmref_parity_")
        try:
            O.run_ref(O.write_ref_spec(case, d, steps=steps, tol_iter=NEWTON_TOL, loop="step"), d, threads=1,
                      timeout=1800)
            rows = O.read_ref_steps(d)
            x0 = O.read_bin(d, "xyz0.f64", np.float64).reshape(-1, 3)
            ref = [O.read_bin(d, f"xyz_{s:03d}.f64", np.float64).reshape(-1, 3) - x0 for s in range(steps)]
        finally:
            shutil.rmtree(d, ignore_errors=True)
        out = {"workload": f"{desc}, first {steps} steps", "workload_short": f"sc3d {size:g} mm, {steps} steps",
               "reference": "oracle/_ref/lpm_ref, 1 thread"}
        for key, prec in (("fp64", lpm.Precision.FP64), ("mixed", lpm.Precision.MIXED)):
            g = lpm.GpuProblem(case.assembly(), undamaged_pt_type=case.undamaged_type, max_iter=case.max_iter,
                               tol_iter=NEWTON_TOL, precision=prec, device=device)
            disp_err, reac_err = 0.0, 0.0
            for s in range(steps):
                ok, st = g.solve_load_step(step_of(case, s))
                u = g.state(("xyz",))["xyz"] - case.xyz
                disp_err = max(disp_err, float(np.linalg.norm(u - ref[s]) / np.linalg.norm(ref[s])))
                rn = rows[s]["reaction_norm"]
                reac_err = max(reac_err, abs(st["reaction_norm"] - rn) / rn)
            g.close()
            out[key] = {"rel_disp_err_vs_reference": disp_err, "rel_reaction_err_vs_reference": reac_err}
        return out
    except Exception as ex:  # the parity figures must not cost the bench line
        return {"error": f"{type(ex).__name__}: {ex}"}


def _steps_header(d):
    with open(os.path.join(d, "steps.txt")) as f:
        head = f.readline()
    m = re.search(r"N (\d+) dim (\d+) setup_s ([0-9.]+)", head)
    return int(m.group(1)), int(m.group(2)), float(m.group(3))


def cpu_baseline(name, size):
    """The reference's CPU path on this host, a bounded sample: the workload's first load step,
    one converged SolverStatic::solveProblemStep call (Newton to the workload's tolerance, the
    reference's CG test) on all host cores, from oracle/_ref/lpm_ref.  Falls back to the
    single-threaded C restatement (assembly + one CG solve) when the reference build is absent."""
    from oracle import oracle as O
    threads = os.cpu_count() or 1
    if O.ref_available():
        d = tempfile.mkdtemp(prefix="lpmref_")
        try:
            O.run_ref(reference_spec(name, size, 1), d, threads=threads, timeout=1800)
            rows = O.read_ref_steps(d)
            n, dim, setup = _steps_header(d)
        finally:
            shutil.rmtree(d, ignore_errors=True)
        it = sum(r["cg_iters"] for r in rows)
        wall = sum(r["wall_s"] for r in rows)
        return {"value": n * dim * it / wall, "unit": UNIT, "cores": threads, "kind": "reference",
                "sample": f"load step 1 of the same workload, one converged solveProblemStep ({rows[0]['newton_solves']} "
                          f"Newton solves, {it} CG iterations, {wall:.1f} s; setup {setup:.1f} s untimed); LPM-CPP "
                          "headers compiled unmodified, MKL replaced by the oracle/shim stand-in",
                "s_per_step": wall, "cg_spmv_s_per_iter": sum(r["spmv_s"] for r in rows) / max(it, 1)}
    case, _ = workload(name, size)
    mat = O.Material(ptype="elastic", plane_stress=case.material.plane_stress, E=case.material.E, mu=case.material.mu,
                     critical_bstrain=case.material.critical_bstrain)
    lat = {0: "sq2d", 1: "hex2d", 2: "sc3d", 3: "fcc3d", 4: "bcc3d"}[int(case.lattice)]
    o = O.OracleProblem(lat, case.radius, case.xyz, mat, types=case.types, cg_maxit=400)
    o.update_geometry()
    o.update_force_state()
    flag = {"x": 0, "y": 1, "z": 2}
    disp = [(case.groups[g], flag[f], v) for g, f, v in case.steps[0][0]]
    o.apply_bc(disp, [])
    t0 = time.perf_counter()
    o.assemble(True)
    o.update_geometry()
    o.update_force_state()
    o.update_rr()
    _, it = o.cg()
    wall = time.perf_counter() - t0
    return {"value": case.n * case.dim * it / wall, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": "C restatement: assembly + 1 CG solve capped at 400 iterations"}


def run_reference(a):
    """The reference arm: oracle/_ref/lpm_ref (LPM-CPP's headers compiled unmodified, MKL replaced
    by the oracle/shim stand-in) runs the same workload on all host cores, W + K converged load
    steps of SolverStatic::solveProblemStep (the loop of solveProblem without the per-step dump),
    the last K timed by the driver's own clock around each call.  The spec is written from the
    workload's definition (reference_spec); nothing of the product is imported or loaded."""
    world, rank, local = dist_setup()
    if rank != 0:
        return
    from oracle import oracle as O
    if not O.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/lpm_ref was not built on this machine"}))
        return
    W, K = a.warmup, a.steps
    threads = os.cpu_count() or 1
    d = tempfile.mkdtemp(prefix="lpmref_arm_")
    try:
        O.run_ref(reference_spec(a.config, a.size, W + K), d, threads=threads, timeout=3600)
        rows = O.read_ref_steps(d)
        n, dim, setup = _steps_header(d)
    finally:
        shutil.rmtree(d, ignore_errors=True)
    timed = rows[W:W + K]
    it = sum(r["cg_iters"] for r in timed)
    wall = sum(r["wall_s"] for r in timed)
    ndof = n * dim
    value = ndof * it / wall
    lat = sorted(r["wall_s"] * 1e3 for r in timed)
    sample = (f"{K} timed of {W + K} converged solveProblemStep calls of the same workload "
              f"({sum(r['newton_solves'] for r in timed) / K:.1f} Newton solves, {it / K:.0f} CG iterations per step); "
              f"setup {setup:.1f} s untimed; LPM-CPP headers compiled unmodified, MKL replaced by the oracle/shim stand-in")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K,
        "warmup": W, "ms_per_step": wall / K * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (reference lattice generator)",
        "config": workload_config(a.config, a.size, n, dim),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "reference", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "solves_per_s": K / wall, "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99))},
        "newton_per_step": sum(r["newton_solves"] for r in timed) / K, "cg_iters_per_step": it / K,
        "parallelism": f"host OpenMP, {threads} threads",
    }), flush=True)


def main():
    a = args_()
    if a.impl == "reference":
        run_reference(a)
    else:
        run_ours(a)


if __name__ == "__main__":
    main()
