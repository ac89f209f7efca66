"""bench.py's reference arm and record (no device).

The reference arm writes its spec for oracle/_ref/lpm_ref from the workload's definition alone
(coordinate conditions for the boundary groups), so that it loads nothing of the product.  These
tests check that the conditions select exactly the groups of the product's workload builders on
the same lattice, that writing the spec imports no product module, and that both arms describe
the workload with the same `config` object.  Where the reference build is present, a short run
of the 6 mm cube through that spec must pick the same particle count as the product's builder.
"""
import importlib
import os
import re
import subprocess
import sys
import tempfile

import numpy as np
import pytest

from _util import CFG, ROOT

sys.path.insert(0, ROOT)
bench = importlib.import_module("bench")


def _groups_from_spec(spec, xyz):
    """Evaluates the spec's `group NAME AXIS OP VALUE ...` conditions on xyz, as the driver does."""
    out = {}
    for line in spec.splitlines():
        t = line.split()
        if not t or t[0] != "group":
            continue
        ok = np.ones(len(xyz), bool)
        for k in range(2, len(t), 3):
            ax, op, v = int(t[k]), t[k + 1], float(t[k + 2])
            ok &= (xyz[:, ax] < v) if op == "<" else (xyz[:, ax] > v)
        out[t[1]] = np.nonzero(ok)[0].astype(np.int32)
    return out


@pytest.mark.parametrize("name,size", [("sc3d", 6.0), ("sc3d", 20.0), ("hex2d", 10.0), ("hex2d", 20.0)])
def test_spec_groups_equal_workload_groups(name, size):
    case, _ = bench.workload(name, size)
    spec = bench.reference_spec(name, size, 3)
    groups = _groups_from_spec(spec, case.xyz)
    assert set(groups) == set(case.groups)
    for g, ids in case.groups.items():
        assert np.array_equal(np.sort(ids), groups[g]), g
    # the same increments on the same groups, every step
    bcs = [tuple(l.split()[1:4]) for l in spec.splitlines() if l.startswith("dispbc")]
    want = [(g, f, repr(float(v))) for g, f, v in case.steps[0][0]]
    assert bcs == want


def test_spec_writing_loads_no_product_module():
    code = ("import sys; sys.path.insert(0, %r); import bench; bench.reference_spec('sc3d', 20.0, 25); "
            "bench.workload_config('sc3d', 20.0, 127500, 3); "
            "assert not [m for m in sys.modules if m.startswith('lpm-cpp_b200')], 'product imported'" % ROOT)
    subprocess.run([sys.executable, "-c", code], check=True)


def test_both_arms_share_the_config_object():
    case, desc = bench.workload("sc3d", 20.0)
    ours = bench.workload_config("sc3d", 20.0, case.n, case.dim)
    ref = bench.workload_config("sc3d", 20.0, 127500, 3)
    assert ours == ref
    assert ours["workload"] == desc


def test_reference_run_through_the_spec_matches_the_workload():
    from oracle import oracle as O
    if not O.ref_available():
        pytest.skip("oracle/_ref/lpm_ref is not built here")
    case, _ = bench.workload("sc3d", 6.0)
    d = tempfile.mkdtemp(prefix="lpmref_spec_")
    O.run_ref(bench.reference_spec("sc3d", 6.0, 1), d, threads=os.cpu_count() or 1, timeout=600)
    n, dim, _ = bench._steps_header(d)
    assert (n, dim) == (case.n, 3)
    xyz0 = O.read_bin(d, "xyz0.f64", np.float64).reshape(-1, 3)
    assert np.array_equal(xyz0, case.xyz)
    rows = O.read_ref_steps(d)
    assert rows[0]["newton_solves"] >= 1 and rows[0]["cuts"] == 0
    typ = O.read_bin(d, "type.i32", np.int32)
    assert np.array_equal(typ, case.types)


def test_compact_record_is_short():
    leg = {"speedup_vs_fp64": 1.2345678, "rel_disp_err_vs_fp64": 1.234567e-8, "dof_iter_per_s": 4.0e9,
           "ms_per_step": 123.456789}
    out = bench._r(bench.compact_legs(leg, None, None, None, None, None, None, None))
    assert out["mixed"]["speedup_vs_fp64"] == 1.235
    assert len(re.sub(r"\s", "", str(out))) < 400
