"""What a proposed starting point can gain, measured on the compiled reference.

A learned warm start that proposes the primal (1-RDM occupations and the
D2ab pair diagonal) and then projects it onto {A x = b} can do no better than
an oracle that proposes the exact converged values.  This test runs the
reference's own boundary-point loop (v2rdm_solver.cc:1778-1908) from

  * the least-norm feasible point (x = A^T w with A A^T w = b, y = z = 0,
    mu = 1; the solver's `start = feasible` option),
  * the exact converged D1 diagonals and D2ab diagonal, projected the same
    way (the best such a proposal can be),
  * the exact converged x itself, with zero duals,
  * the exact converged x and z (y = 0),

and checks that the primal proposals gain under 5 % over the feasible point
while the dual slack z cuts the count by more than half: the state that
decides the boundary-point method's progress is z (y follows from x, z and
mu through the CG step of the first iteration).
"""
import os

import numpy as np
import pytest

from tests.helpers import GOLDEN, load


def _reference_matrix(r):
    import scipy.sparse as sp

    A = np.zeros((r.ncon, r.dimx))
    e = np.zeros(r.dimx)
    for j in range(r.dimx):
        e[j] = 1.0
        A[:, j] = r.Au(e)
        e[j] = 0.0
    return sp.csr_matrix(A)


def _project(A, b, xp):
    """xp plus the least-norm correction onto {A x = b}."""
    import scipy.sparse.linalg as sla

    return xp + sla.lsqr(A, b - A @ xp, atol=1e-15, btol=1e-15, iter_lim=50000)[0]


@pytest.fixture(scope="module")
def case(ref):
    from v2rdm_casscf_b200.hamiltonian import synthetic

    g = load(os.path.join(GOLDEN, "solve_synthetic_n4_s0.npz"))
    a = synthetic(4, 0)
    r = ref.RefSolver([4], [a.nb], positivity="DQG", r_convergence=1e-6, e_convergence=1e-7)
    r.set_integrals(a.oei_packed, a.qmo, a.nq)
    r.build_constraints()
    A = _reference_matrix(r)
    return r, A, r.get("b"), g


def _solve(r, x, y, z):
    r.set("x", x)
    r.set("y", y)
    r.set("z", z)
    return r.solve(mu=1.0)


def test_primal_proposals_gain_nothing_over_feasible_start(case):
    r, A, b, g = case
    X, Z = g["x"], g["z"]
    y0, z0 = np.zeros(r.ncon), np.zeros(r.dimx)
    feas = _solve(r, _project(A, b, z0), y0, z0)
    assert feas["converged"] and abs(feas["e_primal"] - float(g["e_primal"])) <= 1e-6

    n, g2 = 4, 16
    d1a, d1b, d2ab = r.offsets("d1a")[0], r.offsets("d1b")[0], r.offsets("d2ab")[0]
    xp = np.zeros(r.dimx)
    for i in range(n):
        xp[d1a + i * n + i] = X[d1a + i * n + i]
        xp[d1b + i * n + i] = X[d1b + i * n + i]
    for k in range(g2):
        xp[d2ab + k * g2 + k] = X[d2ab + k * g2 + k]
    diag = _solve(r, _project(A, b, xp), y0, z0)
    full_x = _solve(r, X, y0, z0)
    with_z = _solve(r, X, y0, Z)
    for out in (diag, full_x, with_z):
        assert out["converged"] and abs(out["e_primal"] - float(g["e_primal"])) <= 1e-6
    # the best primal proposal gains under 5 % ...
    assert diag["oiter"] >= 0.95 * feas["oiter"]
    assert full_x["oiter"] >= 0.95 * feas["oiter"]
    # ... while the converged dual slack more than halves the count
    assert with_z["oiter"] <= 0.5 * feas["oiter"]
