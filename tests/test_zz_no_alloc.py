"""The allocation-free CG entry point (lpmgpu_cg_bsr_noalloc).

It serves callers that cannot allocate device memory: a plugin inside a host program that owns
all device memory through its own pool or arena, and latency-bound loops that cannot afford
cudaMalloc/cudaFree, which may synchronise the device.  The tests build a stiffness system with
the regular handle, hand the same matrix (as device block-CSR) and right-hand side to the
allocation-free entry point through the C ABI, and check two consecutive calls against the
handle's own linear solve (lpmgpu_solve_linear) and against the CPU oracle's CG on the same
system, at the tolerance of the other linear-solve tests.  One case runs on a caller's stream
with work already queued on it and a grid of many blocks.  Further cases check that a solve
stopped by its iteration cap, one fed NaN, and one that breaks down (p.Ap == 0) report their
status instead of success.  This file is collected last so that a run stopping at the first
failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

from _util import CFG, LPM, gpu_problem, oracle_problem, oracle_step_args, rel

pytestmark = pytest.mark.gpu

SOLVE_TOL = 1e-9  # same bar as test_gpu_parity.test_linear_solve
CASES = {
    "hex": lambda: CFG.hex_plate(size=4.0, radius=0.1, steps=1, total_disp=0.001),
    "sc": lambda: CFG.sc_cube(size=2.4, radius=0.2, steps=1, total_disp=0.001),
    # 15,625 particles, 46,875 unknowns: 16 blocks of the cooperative grid
    "sc10": lambda: CFG.sc_cube(size=10.0, radius=0.2, steps=1, total_disp=0.001),
}


def _system(case):
    g = gpu_problem(case, cg_rtol=1e-24, cg_atol=0.0)
    g.apply_load_step(case.load_step(0))
    g.assemble(True)
    g.update_force_state()
    g.update_rr()
    x_ref, st = g.solve_linear()
    Kp, IK, JK, K = g.export_csr()
    return g, x_ref, IK, JK, K, g.residual()


def _oracle_solution(case):
    o = oracle_problem(case, cg_rtol=1e-24, cg_atol=0.0)
    o.update_geometry()
    o.update_force_state()
    o.apply_bc(*oracle_step_args(case, 0))
    o.assemble(True)
    o.update_geometry()
    o.update_force_state()
    o.update_rr()
    xo, _ = o.cg()
    return xo


def _bsr(IK, JK, K, n, dim):
    import scipy.sparse as sp
    N = n * dim
    # reference layout: 1-based upper CSR, IK[N+1] row starts, JK columns (stiffness.h:24-26)
    U = sp.csr_matrix((K, JK - 1, IK - 1), shape=(N, N))
    A = (U + U.T - sp.diags(U.diagonal())).tocsr()
    B = A.tobsr(blocksize=(dim, dim))
    B.sort_indices()
    return (B.indptr.astype(np.int32), B.indices.astype(np.int32),
            np.ascontiguousarray(B.data.reshape(-1), dtype=np.float64))


def _call(L, dim, n, d_rp, d_col, d_val, d_b, d_x, rtol, atol, maxit, stream):
    it = C.c_int64(-1)
    status = L.lpmgpu_cg_bsr_noalloc(dim, n, C.c_void_p(d_rp.data_ptr()), C.c_void_p(d_col.data_ptr()),
                                     C.c_void_p(d_val.data_ptr()), C.c_void_p(d_b.data_ptr()),
                                     C.c_void_p(d_x.data_ptr()), rtol, atol, maxit, stream, C.byref(it))
    return status, it.value


def _device_system(torch, case):
    g, x_ref, IK, JK, K, b = _system(case)
    n, dim = g.n, g.dim
    rowptr, col, val = _bsr(np.asarray(IK), np.asarray(JK), np.asarray(K), n, dim)
    assert len(rowptr) == n + 1
    dev = torch.device("cuda", 0)
    d = [torch.from_numpy(a).to(dev) for a in (rowptr, col, val, np.ascontiguousarray(b))]
    return g, x_ref, n, dim, d


@pytest.mark.parametrize("lat,user_stream", [("hex", False), ("sc", False), ("sc10", True)])
def test_noalloc_matches_solve_linear_and_oracle_twice(lat, user_stream):
    torch = pytest.importorskip("torch")
    case = CASES[lat]()
    g, x_ref, n, dim, (d_rp, d_col, d_val, d_b) = _device_system(torch, case)
    x_oracle = _oracle_solution(case)
    assert rel(x_ref, x_oracle) <= SOLVE_TOL
    L = LPM.lib()
    stream = torch.cuda.Stream() if user_stream else None
    for call in range(2):
        torch.cuda.synchronize()
        if stream is not None:
            # work queued on the caller's stream ahead of the solve: a fresh right-hand side copy
            # and the output poisoned with NaN, both of which the solve must see in stream order
            with torch.cuda.stream(stream):
                d_rhs = d_b.clone()
                d_x = torch.full((n * dim,), float("nan"), dtype=torch.float64, device=d_b.device)
            status, it = _call(L, dim, n, d_rp, d_col, d_val, d_rhs, d_x, 1e-24, 0.0, 0, C.c_void_p(stream.cuda_stream))
        else:
            d_x = torch.full((n * dim,), float("nan"), dtype=torch.float64, device=d_b.device)
            torch.cuda.synchronize()
            status, it = _call(L, dim, n, d_rp, d_col, d_val, d_b, d_x, 1e-24, 0.0, 0, None)
        assert status == 0, L.lpmgpu_last_error()
        x = d_x.cpu().numpy()
        assert it > 0
        e = rel(x, x_ref)
        assert e <= SOLVE_TOL, f"call {call}: relative difference to lpmgpu_solve_linear {e}"
        e = rel(x, x_oracle)
        assert e <= SOLVE_TOL, f"call {call}: relative difference to the oracle's CG {e}"
    g.close()


def test_noalloc_reports_cap_nan_and_breakdown():
    torch = pytest.importorskip("torch")
    case = CASES["sc"]()
    g, _, n, dim, (d_rp, d_col, d_val, d_b) = _device_system(torch, case)
    L = LPM.lib()
    d_x = torch.zeros(n * dim, dtype=torch.float64, device=d_b.device)
    # the cap: 3 iterations cannot meet the tolerance
    status, it = _call(L, dim, n, d_rp, d_col, d_val, d_b, d_x, 1e-24, 0.0, 3, None)
    assert status == LPM.ERR_CG_MAXIT, (status, L.lpmgpu_last_error())
    assert it == 3
    # NaN in the right-hand side never meets the test and ends at the cap
    d_nan = d_b.clone()
    d_nan[0] = float("nan")
    status, it = _call(L, dim, n, d_rp, d_col, d_val, d_nan, d_x, 1e-24, 0.0, 5, None)
    assert status == LPM.ERR_CG_MAXIT, (status, L.lpmgpu_last_error())
    # a zero matrix: p.Ap == 0 at the first iteration
    d_zero = torch.zeros_like(d_val)
    status, it = _call(L, dim, n, d_rp, d_col, d_zero, d_b, d_x, 1e-24, 0.0, 0, None)
    assert status == LPM.ERR_CG_BREAKDOWN, (status, L.lpmgpu_last_error())
    assert it == 0
    # the entry point is usable afterwards
    status, it = _call(L, dim, n, d_rp, d_col, d_val, d_b, d_x, 1e-24, 0.0, 0, None)
    assert status == 0 and it > 0
    g.close()


def test_noalloc_rejects_sizes_beyond_its_scratch():
    L = LPM.lib()
    one = C.c_void_p(1)  # never dereferenced: the size check comes first
    it = C.c_int64(0)
    assert L.lpmgpu_cg_bsr_noalloc(3, 100000, one, one, one, one, one, 1e-12, 1e-12, 0, None, C.byref(it)) == 1
    assert b"262144" in L.lpmgpu_last_error()
