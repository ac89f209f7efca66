"""The reference's one known-answer test: examples/ex7_convergence_beam.cpp, a plane-strain
hexagonal cantilever beam with the analytic displacement of Solution::computeSolBeam001 and the
relative L2 error of computeL2Error (include/solution.h:27-63), evaluated as coded (its u1 term
holds the integer division 1 / 6, which is 0: solution.h:41).  The reference's own hot path and
the CPU oracle solve the example's beam with the example's tolerances; their displacements and
L2 errors must agree, and the error must be that of a converged LPM solution of this beam."""
import math
import os

import numpy as np
import pytest

from _util import CFG, O, oracle_problem, oracle_step_args, rel


def beam_l2_error(xyz0, xyz, L, D, P, E, mu):
    """Solution::computeSolBeam001 + computeL2Error, in the reference's operator order."""
    G = E / 2 / (1 + mu)
    I = D * D * D / 12
    err_sq = exact_sq = 0.0
    for (x, y, _), (X, Y, _) in zip(xyz0, xyz):
        ax, ay = X - x, Y - y
        u1 = (-P * (x * x) * y / 2 / E / I + P * math.pow(y, 3) * ((1 // 6) / G / I - mu / 6 / E / I)
              + y * (P * L * L / 2 / E / I - P * D * D / 8 / G / I))
        u2 = (mu * P * x * (y * y) / 2 / E / I + P * math.pow(x, 3) / 6 / E / I - P * L * L * x / 2 / E / I
              + P * L * L * L / 3 / E / I)
        for ex, ap in ((u1, ax), (u2, ay)):
            err_sq += (ex - ap) * (ex - ap)
            exact_sq += ex * ex
    return -1.0 if exact_sq < 1e-6 else math.sqrt(err_sq / exact_sq)


# computeL2Error of the reference's own solution of the example's beam (oracle/_ref/lpm_ref, this
# file's test below): the known answer the oracle must reproduce
BEAM_L2_REFERENCE = 0.0762656679707


def _oracle_beam():
    case = CFG.cantilever_beam()
    o = oracle_problem(case)
    o.update_geometry()
    o.update_force_state()
    ok, st = o.solve_load_step(*oracle_step_args(case, 0))
    assert ok and st["newton_solves"] == 2
    m = case.meta
    args = (m["length"], m["depth"], m["force"], case.material.E, case.material.mu)
    return case, o.state()["xyz"], args


def test_oracle_beam_known_answer():
    case, x_o, args = _oracle_beam()
    assert case.n == 6000
    assert abs(beam_l2_error(case.xyz, x_o, *args) - BEAM_L2_REFERENCE) <= 1e-8 * BEAM_L2_REFERENCE


@pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref/lpm_ref not built (make -C oracle ref)")
def test_beam_known_answer_matches_the_reference_run(tmp_path):
    case, x_o, args = _oracle_beam()
    d = str(tmp_path / "ref")
    os.makedirs(d)
    O.run_ref(O.write_ref_spec(case, d, loop="ref"), d, threads=1)
    assert np.array_equal(O.read_bin(d, "xyz0.f64", np.float64).reshape(-1, 3), case.xyz)
    x_ref = O.read_bin(d, "xyz_000.f64", np.float64).reshape(-1, 3)
    e_ref = beam_l2_error(case.xyz, x_ref, *args)
    # both stop at the example's own tolerances (Newton 1e-5, CG 1e-12 on squared norms)
    assert rel(x_o - case.xyz, x_ref - case.xyz) <= 1e-8
    assert abs(beam_l2_error(case.xyz, x_o, *args) - e_ref) <= 1e-8 * e_ref
    assert abs(e_ref - BEAM_L2_REFERENCE) <= 1e-8 * BEAM_L2_REFERENCE
