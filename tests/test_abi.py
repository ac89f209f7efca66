"""The C-ABI library (no compute without a GPU): it loads, exports every symbol that
include/lpmgpu.h declares, rejects bad input with status codes, and refuses to run without a
CUDA device instead of falling back to the CPU."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from _util import CFG, LPM, ROOT
from conftest import cuda_available

HEADER = os.path.join(ROOT, "include", "lpmgpu.h")


def declared():
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?[\w]+\s*\*?\s*(lpmgpu_\w+)\s*\(", txt, flags=re.M)))


def test_header_declares_entry_points():
    names = declared()
    assert "lpmgpu_create" in names and "lpmgpu_solve_load_step" in names
    assert len(names) >= 20


def test_library_exports_every_declared_symbol():
    lib = C.CDLL(LPM.LIB_PATH)
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing
    assert sorted(LPM.EXPORTS) == declared(), "lpm.py binds exactly the declared symbols"


def test_version_and_status_strings():
    L = LPM.lib()
    assert b"sm_100a" in L.lpmgpu_version()
    assert L.lpmgpu_status_string(0) == b"ok"
    assert L.lpmgpu_status_string(4).startswith(b"Newton")


def test_invalid_arguments_are_rejected():
    L = LPM.lib()
    h = C.c_void_p()
    assert L.lpmgpu_create(None, C.byref(h)) == 1
    d = LPM.Desc()
    d.n = 0
    assert L.lpmgpu_create(C.byref(d), C.byref(h)) == 1
    cnt = C.c_int64()
    box = np.zeros(6)
    ang = np.zeros(3)
    assert L.lpmgpu_generate_lattice(9, 0.1, box.ctypes.data_as(C.POINTER(C.c_double)), 0,
                                     ang.ctypes.data_as(C.POINTER(C.c_double)), None, 0, C.byref(cnt)) == 1
    assert L.lpmgpu_destroy(None) == 1
    assert L.lpmgpu_solve_load_step(None, None, None) == 1
    assert L.lpmgpu_batch_create(0, None) == 1
    assert L.lpmgpu_batch_destroy(None) == 1
    assert L.lpmgpu_batch_add(None, None, None, 0, None) == 1
    assert L.lpmgpu_batch_round(None, None) == 1
    assert L.lpmgpu_server_create(0, 0, None) == 1
    assert L.lpmgpu_server_submit(None, None, None, 0, None) == 1
    assert L.lpmgpu_estimate_bytes(None, None) == 1
    assert L.lpmgpu_autotune(None, 10, None) == 1
    assert L.lpmgpu_set_cg_grid(None, 4) == 1


@pytest.mark.skipif(cuda_available(), reason="checks the no-device path")
def test_no_device_fails_loudly():
    case = CFG.hex_plate(size=1.0, radius=0.1, steps=1)
    with pytest.raises(LPM.LpmGpuError) as e:
        LPM.GpuProblem(case.assembly())
    assert e.value.status in (2, 11)
    with pytest.raises(LPM.LpmGpuError) as e:
        LPM.Batch()
    assert e.value.status in (2, 11)


def test_generators_are_host_side():
    """Lattice generation needs no device (utilities.h restated on the host)."""
    cell = LPM.UnitCell(LPM.LatticeType.SimpleCubic3D, 0.2)
    x = LPM.createCuboidSC3D([0, 2, 0, 2, 0, 2], cell)
    from oracle import oracle as O
    assert len(x) > 100 and np.array_equal(x, O.generate("sc3d", 0.2, [0, 2, 0, 2, 0, 2]))


def test_estimate_counts_the_nonlocal_lists():
    """The admission estimate (lpmgpu_estimate_bytes, host arithmetic) grows by at least the
    device bytes of the nonlocal neighbour lists the search will hold: 4 per neighbour (the
    particle itself included) plus an offset and a rate per particle."""
    from scipy.spatial import cKDTree
    for c in (CFG.edamage_plate(), CFG.edamage_plate(size=3.0, cutoff_ratio=3.0)):
        a = c.assembly()
        with_nl = LPM.Server.estimate_bytes(a)
        a.nonlocal_cutoff_ratio = 0.0
        without = LPM.Server.estimate_bytes(a)
        R = c.nonlocal_cutoff_ratio * c.material.nonlocal_L
        pairs = sum(len(v) for v in cKDTree(c.xyz).query_ball_point(c.xyz, R * (1 - 1e-12)))
        assert with_nl - without >= 4 * pairs + 12 * c.n


def test_tune_result_layout_matches_the_header():
    """lpmgpu_tune_result: four int32 then LPMGPU_TUNE_MAX int32 grids and doubles."""
    txt = open(HEADER).read()
    m = re.search(r"#define LPMGPU_TUNE_MAX (\d+)", txt)
    assert m and int(m.group(1)) == 8
    assert LPM.TuneResult.us_per_iter.offset == 4 * 4 + 8 * 4
    assert C.sizeof(LPM.TuneResult) == 4 * 4 + 8 * 4 + 8 * 8


def test_estimate_counts_explicit_nonlocal_lists():
    """Nonlocal lists handed over in lpmgpu_desc (nonlocal_count / nonlocal_ids, as the C++
    drop-ins pass an Assembly's own) count exactly in the admission estimate: 4 bytes an entry
    plus an offset and a rate per particle."""
    c = CFG.hex_plate(size=2.0, radius=0.1)
    a = c.assembly()
    d, keep = LPM._pack_desc(a)
    base = C.c_int64()
    assert LPM.lib().lpmgpu_estimate_bytes(C.byref(d), C.byref(base)) == 0
    cnt = np.full(c.n, 7, np.int32)
    ids = np.zeros(7 * c.n, np.int32)
    d.nonlocal_count = cnt.ctypes.data_as(C.POINTER(C.c_int32))
    d.nonlocal_ids = ids.ctypes.data_as(C.POINTER(C.c_int32))
    with_lists = C.c_int64()
    assert LPM.lib().lpmgpu_estimate_bytes(C.byref(d), C.byref(with_lists)) == 0
    assert with_lists.value - base.value == 4 * 7 * c.n + 12 * c.n
