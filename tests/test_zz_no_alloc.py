"""The allocation-free CG entry point (lpmgpu_cg_bsr_noalloc).

It serves callers that cannot allocate device memory: code under CUDA graph capture and hosts
whose device memory belongs to an external pool.  The test builds a stiffness system with the
regular handle, hands the same matrix (as device block-CSR) and right-hand side to the
allocation-free entry point through the C ABI, and checks two consecutive calls against the
handle's own linear solve (lpmgpu_solve_linear) at the tolerance of the other linear-solve
tests.  This file is collected last so that a run stopping at the first failure has already
run every other test.
"""
import ctypes as C

import numpy as np
import pytest

from _util import CFG, LPM, gpu_problem, rel

pytestmark = pytest.mark.gpu

SOLVE_TOL = 1e-9  # same bar as test_gpu_parity.test_linear_solve


def _system(case):
    g = gpu_problem(case, cg_rtol=1e-24, cg_atol=0.0)
    g.apply_load_step(case.load_step(0))
    g.assemble(True)
    g.update_force_state()
    g.update_rr()
    x_ref, st = g.solve_linear()
    Kp, IK, JK, K = g.export_csr()
    return g, x_ref, IK, JK, K, g.residual()


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


@pytest.mark.parametrize("lat", ["hex", "sc"])
def test_noalloc_matches_solve_linear_twice(lat):
    torch = pytest.importorskip("torch")
    if lat == "hex":
        case = CFG.hex_plate(size=4.0, radius=0.1, steps=1, total_disp=0.001)
    else:
        case = CFG.sc_cube(size=2.4, radius=0.2, steps=1, total_disp=0.001)
    g, x_ref, IK, JK, K, b = _system(case)
    n, dim = g.n, g.dim
    rowptr, col, val = _bsr(np.asarray(IK), np.asarray(JK), np.asarray(K), n, dim)
    assert len(rowptr) == n + 1
    dev = torch.device("cuda", 0)
    d_rp = torch.from_numpy(rowptr).to(dev)
    d_col = torch.from_numpy(col).to(dev)
    d_val = torch.from_numpy(val).to(dev)
    d_b = torch.from_numpy(np.ascontiguousarray(b)).to(dev)
    L = LPM.lib()
    for call in range(2):
        d_x = torch.full((n * dim,), float("nan"), dtype=torch.float64, device=dev)
        torch.cuda.synchronize()
        it = C.c_int64(-1)
        status = L.lpmgpu_cg_bsr_noalloc(dim, n, C.c_void_p(d_rp.data_ptr()), C.c_void_p(d_col.data_ptr()),
                                         C.c_void_p(d_val.data_ptr()), C.c_void_p(d_b.data_ptr()),
                                         C.c_void_p(d_x.data_ptr()), 1e-24, 0.0, 0, None, C.byref(it))
        assert status == 0, L.lpmgpu_last_error()
        x = d_x.cpu().numpy()
        assert it.value > 0
        e = rel(x, x_ref)
        assert e <= SOLVE_TOL, f"call {call}: relative difference {e}"
    g.close()


def test_noalloc_rejects_sizes_beyond_its_scratch():
    L = LPM.lib()
    one = C.c_void_p(1)  # never dereferenced: the size check comes first
    it = C.c_int64(0)
    assert L.lpmgpu_cg_bsr_noalloc(3, 100000, one, one, one, one, one, 1e-12, 1e-12, 0, None, C.byref(it)) == 1
    assert b"262144" in L.lpmgpu_last_error()
