"""Per-step dump output (Assembly::writeDump, include/assembly.h:310-335): the native writer of
the C ABI against the reference's own dump files and against the printf conversions, and the
device path (pinned copy + writer thread) against the host formatter."""
import os

import numpy as np
import pytest

from _util import CFG, LPM
from oracle import oracle as O


def _ref_dump_case(case, tmp_path, name):
    """Runs the reference's SolverStatic::solveProblem step by step with a dump file; returns the
    dump text and the per-step state binaries' directory."""
    d = str(tmp_path / name)
    os.makedirs(d)
    spec = O.write_ref_spec(case, d, loop="ref", cg_tol=(1e-24, 0.0), tol_iter=1e-9)
    dump = os.path.join(d, "ref.dump")
    O.run_ref(spec + f"\ndumpfile {dump}\n", d, threads=1)
    return open(dump, "rb").read(), d


@pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref/lpm_ref not built (make -C oracle ref)")
@pytest.mark.parametrize("which", ["hex_elastic", "sc_j2"])
def test_format_dump_reproduces_the_reference_dump(tmp_path, which):
    """The reference's own writeDump output, byte for byte, from the same per-step values."""
    if which == "hex_elastic":
        case = CFG.hex_plate(size=1.6, radius=0.1, steps=2, total_disp=0.002)
    else:
        case = CFG.sc_cube(size=1.6, radius=0.2, steps=2, total_disp=0.006, ptype=LPM.ParticleType.J2Plasticity,
                           j2=(200.0, 0.0, 38714.0, 10.0))
    text, d = _ref_dump_case(case, tmp_path, which)
    out = str(tmp_path / "ours.dump")
    n = case.n
    nsv = 7 if which == "sc_j2" else 1
    for s in range(len(case.steps)):
        tag = "%03d" % s
        xyz = O.read_bin(d, f"xyz_{tag}.f64", np.float64).reshape(n, 3)
        sv = O.read_bin(d, f"state_var_{tag}.f64", np.float64).reshape(n, -1)
        assert sv.shape[1] == nsv
        LPM.format_dump(out, s, case.box, xyz, case.xyz, O.read_bin(d, f"stress_{tag}.f64", np.float64),
                        O.read_bin(d, f"damage_{tag}.f64", np.float64),
                        O.read_bin(d, f"damage_visual_{tag}.f64", np.float64), sv, type=case.types, threads=3)
    if which == "sc_j2":
        assert np.any(sv[:, 0] > 0), "the J2 cube must yield so that state_var[0] is exercised"
    assert open(out, "rb").read() == text


def test_format_dump_conversions_and_threads(tmp_path):
    """Edge values (signed zeros, tiny and huge magnitudes, three-digit exponents, ties at the
    fourth digit) convert as printf's %.4e / %8.8f do, and the chunked parallel formatting gives
    the same bytes for any thread count."""
    rng = np.random.default_rng(7)
    n = 9001
    special = np.array([0.0, -0.0, 1e-300, -1e300, 5e-324, 1.23455, 1.23465, 9.99995e7, -2.5e-5, 123456789.0])
    def field(k):
        v = rng.standard_normal(n * k) * 10.0 ** rng.integers(-12, 12, n * k)
        v[: len(special)] = special[: min(len(special), n * k)]
        return v
    xyz, xyz0, st, dmg, dv, sv = field(3), field(3), field(6), field(1), field(1), field(1)
    box = np.array([-1.0, 2.5, -0.125, 1e3, 0.0, -0.0])
    types = rng.integers(-3, 5, n).astype(np.int32)
    paths = []
    for threads in (1, 2, 7, 0):
        p = str(tmp_path / f"t{threads}.dump")
        LPM.format_dump(p, 12, box, xyz, xyz0, st, dmg, dv, sv, type=types, threads=threads)
        paths.append(p)
    texts = [open(p, "rb").read() for p in paths]
    assert all(t == texts[0] for t in texts[1:])
    x, x0, s = xyz.reshape(n, 3), xyz0.reshape(n, 3), st.reshape(n, 6)
    lines = ["ITEM: TIMESTEP", "12", "ITEM: NUMBER OF ATOMS", str(n), "ITEM: BOX BOUNDS pp pp pp"]
    lines += ["%8.8f %8.8f" % (box[2 * k], box[2 * k + 1]) for k in range(3)]
    lines.append("ITEM: ATOMS id type x y z dx dy dz s11 s22 s33 s23 s13 s12 damage damage_visual state_var[0] ")
    for i in range(n):
        u = x[i] - x0[i]
        vals = [*x[i], *u, *s[i], dmg[i], dv[i], sv[i]]
        lines.append("%d %d " % (i, types[i]) + " ".join("%.4e" % v for v in vals))
    assert texts[0].decode() == "\n".join(lines) + "\n"


def test_format_dump_rejects_bad_arguments(tmp_path):
    L = LPM.lib()
    box = np.zeros(6)
    assert L.lpmgpu_format_dump(None, 0, 0, None, LPM._dp(box), None, None, None, None, None, None, 1, 1) != 0
    assert L.lpmgpu_format_dump(str(tmp_path / "x").encode(), 0, 4, None, LPM._dp(box), None, None, None, None, None,
                                None, 1, 1) != 0
    with pytest.raises(LPM.LpmGpuError):
        LPM.format_dump(str(tmp_path / "no_such_dir" / "x.dump"), 0, box, np.zeros((1, 3)), np.zeros((1, 3)),
                        np.zeros(6), np.zeros(1), np.zeros(1), np.zeros(1))


@pytest.mark.gpu
def test_device_dump_matches_host_formatter(tmp_path):
    """lpmgpu_dump_write (async, two steps queued behind the solves, then flushed; and sync) writes
    what the host formatter writes for the state read back after each step."""
    case = CFG.hex_plate(size=2.0, radius=0.1, steps=3, total_disp=0.003)
    g = LPM.GpuProblem(case.assembly(), tol_iter=1e-9, cg_rtol=1e-24, cg_atol=0.0, device=0)
    dev_async, dev_sync, host = (str(tmp_path / f) for f in ("a.dump", "s.dump", "h.dump"))
    for s in range(len(case.steps)):
        ok, _ = g.solve_load_step(case.load_step(s))
        assert ok
        g.dump_write(dev_async, s, case.box, threads=2, async_=True)
        g.dump_write(dev_sync, s, case.box, threads=1, async_=False)
        st = g.state(("xyz", "stress", "damage", "damage_visual", "state_var"))
        LPM.format_dump(host, s, case.box, st["xyz"], case.xyz, st["stress"], st["damage"], st["damage_visual"],
                        st["state_var"], type=case.types)
    g.dump_flush()
    ref = open(host, "rb").read()
    assert open(dev_async, "rb").read() == ref
    assert open(dev_sync, "rb").read() == ref
    g.close()
