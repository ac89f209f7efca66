"""Host-checkable parts of the direct solver and of the nonlocal search (no device).
- The band Cholesky core of lpm-cpp_b200/csrc/band_chol.cuh, compiled for the host by a harness
  that runs it in the device driver's order and thread decomposition (tests/native/band_check.cpp),
  against numpy on random banded SPD matrices.
- The reverse Cuthill-McKee ordering (lpmgpu_band_order, host only) on the particle connection
  graphs of the reference's lattices.
- The cell-grid nonlocal search of lpm-cpp_b200/csrc/nonlocal_grid.cuh (tests/native/
  nlgrid_check.cpp) against the all-pairs search."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

from _util import CFG, LPM, ROOT, oracle_problem

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("band") / "band_check")
    subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-I", os.path.join(ROOT, "lpm-cpp_b200", "csrc"),
                    os.path.join(HERE, "native", "band_check.cpp"), "-o", exe], check=True)
    return exe


def _banded_spd(n, kd, seed, shift=1.0):
    rng = np.random.default_rng(seed)
    A = np.zeros((n, n))
    for i in range(n):
        for j in range(max(0, i - kd), i):
            A[i, j] = A[j, i] = rng.uniform(-1, 1)
    A += np.diag(np.abs(A).sum(axis=1) + shift)  # diagonally dominant: positive definite
    return A


def _run(exe, tmp, A, kd, nb, b):
    n = len(A)
    ldab = kd + 1
    AB = np.zeros((n, ldab))  # column j at AB[j]
    for j in range(n):
        for i in range(j, min(n, j + kd + 1)):
            AB[j, i - j] = A[i, j]
    fin, fout = str(tmp / "in.bin"), str(tmp / "out.bin")
    with open(fin, "wb") as f:
        np.array([n, kd, nb], np.int64).tofile(f)
        AB.tofile(f)
        np.asarray(b, np.float64).tofile(f)
    subprocess.run([exe, fin, fout], check=True)
    raw = open(fout, "rb").read()
    x = np.frombuffer(raw[:8 * n], np.float64)
    L = np.frombuffer(raw[8 * n:8 * n + 8 * n * ldab], np.float64).reshape(n, ldab)
    fail = int(np.frombuffer(raw[-4:], np.int32)[0])
    return x, L, fail


@pytest.mark.parametrize("n,kd,nb", [(100, 7, 32), (100, 40, 32), (97, 96, 32), (64, 200, 16), (150, 3, 8),
                                     (33, 1, 32), (1, 0, 32), (70, 31, 32)])
def test_band_cholesky_solves_like_numpy(harness, tmp_path, n, kd, nb):
    kd_eff = min(kd, n - 1)
    A = _banded_spd(n, kd_eff, seed=n * 1000 + kd)
    b = np.random.default_rng(7).standard_normal(n)
    x, L, fail = _run(harness, tmp_path, A, kd_eff, nb, b)
    assert fail == 0
    xr = np.linalg.solve(A, b)
    assert np.linalg.norm(x - xr) <= 1e-12 * np.linalg.norm(xr)
    Lr = np.linalg.cholesky(A)
    for j in range(n):
        col = Lr[j:min(n, j + kd_eff + 1), j]
        assert np.allclose(L[j, :len(col)], col, rtol=1e-12, atol=1e-14)


def test_band_cholesky_reports_a_non_positive_pivot(harness, tmp_path):
    A = _banded_spd(50, 5, seed=3)
    A[20, 20] = -1.0
    _, _, fail = _run(harness, tmp_path, A, 5, 16, np.ones(50))
    assert fail == 21  # 1-based column of the first pivot that is not positive


def _rcm(start, adj):
    L = LPM.lib()
    n = len(start) - 1
    rank = np.zeros(n, np.int32)
    bw = C.c_int64()
    s = np.ascontiguousarray(start, np.int32)
    a = np.ascontiguousarray(adj, np.int32)
    st = L.lpmgpu_band_order(n, s.ctypes.data_as(C.POINTER(C.c_int32)), a.ctypes.data_as(C.POINTER(C.c_int32)),
                             rank.ctypes.data_as(C.POINTER(C.c_int32)), C.byref(bw))
    return st, rank, bw.value


@pytest.mark.parametrize("which", ["hex", "sc"])
def test_rcm_order_on_the_connection_graph(which):
    case = CFG.hex_plate(size=3.0, radius=0.1) if which == "hex" else CFG.sc_cube(size=2.0, radius=0.2)
    o = oracle_problem(case)
    nconn, _, conns = o.conns()
    start = np.concatenate([[0], np.cumsum(nconn)]).astype(np.int32)
    st, rank, bw = _rcm(start, conns)
    assert st == 0
    assert np.array_equal(np.sort(rank), np.arange(case.n))
    owner = np.repeat(np.arange(case.n), nconn)
    assert bw == np.abs(rank[owner] - rank[conns]).max()
    natural = np.abs(owner - conns).max()
    assert bw <= natural  # the narrower of RCM and the generator's own order
    # a plate lying across its rows: the generator's order is wide, RCM narrows it
    rot = np.argsort(case.xyz[:, 0] * 1e3 + case.xyz[:, 1], kind="stable")  # column-major renumbering
    inv = np.empty_like(rot)
    inv[rot] = np.arange(case.n)
    nb_start = np.concatenate([[0], np.cumsum(nconn[rot])]).astype(np.int32)
    adj2 = np.concatenate([inv[conns[start[i]:start[i + 1]]] for i in rot]).astype(np.int32)
    st2, rank2, bw2 = _rcm(nb_start, adj2)
    assert st2 == 0 and bw2 <= bw + bw // 2


def test_rcm_order_handles_components_and_rejects_bad_graphs():
    # two disjoint paths 0-1-2 and 3-4
    start = np.array([0, 1, 3, 4, 5, 6], np.int32)
    adj = np.array([1, 0, 2, 1, 4, 3], np.int32)
    st, rank, bw = _rcm(start, adj)
    assert st == 0 and sorted(rank) == list(range(5)) and bw == 1
    assert _rcm(np.array([0, 1], np.int32), np.array([5], np.int32))[0] == 1


# ---- the cell-grid nonlocal search (lpm-cpp_b200/csrc/nonlocal_grid.cuh), host-compiled
@pytest.fixture(scope="module")
def nlgrid(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("nlgrid") / "nlgrid_check")
    subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-I", os.path.join(ROOT, "lpm-cpp_b200", "csrc"),
                    os.path.join(HERE, "native", "nlgrid_check.cpp"), "-o", exe], check=True)
    return exe


@pytest.mark.parametrize("which,max_cells", [("hex", 1 << 26), ("sc", 1 << 26), ("random", 1 << 26),
                                             ("random", 8), ("hex", 1)])
def test_grid_nonlocal_search_finds_the_all_pairs_lists(nlgrid, tmp_path, which, max_cells):
    """Every particle's list from the cells around it, sorted, equals the all-pairs list; also
    when the grid is capped to a few cells (wider cells) or to one."""
    if which == "hex":
        xyz, rc = CFG.hex_plate(size=3.0, radius=0.1).xyz, 0.45
    elif which == "sc":
        xyz, rc = CFG.sc_cube(size=2.0, radius=0.2).xyz, 0.9
    else:
        xyz, rc = np.random.default_rng(5).uniform(-1.0, 2.0, (700, 3)), 0.37
    p = str(tmp_path / "in.bin")
    with open(p, "wb") as f:
        np.array([len(xyz)], np.int64).tofile(f)
        np.array([rc], np.float64).tofile(f)
        np.ascontiguousarray(xyz, np.float64).tofile(f)
    out = subprocess.run([nlgrid, p, str(max_cells)], check=True, capture_output=True, text=True).stdout.split()
    bad, pairs = int(out[0]), int(out[1])
    assert bad == 0
    d = np.linalg.norm(xyz[:, None, :] - xyz[None, :, :], axis=2)
    assert pairs == int((d < rc).sum())
