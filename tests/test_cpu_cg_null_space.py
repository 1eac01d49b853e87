"""Why the product's CG stops on residual growth: A A^T is singular.

The reference's constraint rows are linearly dependent (A^T has a null space
of dimension 73 at n = 4, DQG), so a CG right-hand side with a component in
that null space above the CG tolerance cannot be met.  The plain CG of
cg_solver.cc:125-177 then diverges and y grows without bound (the way an
iterate can turn non-finite); the product stops instead when r.r rises
past 1e4 times its smallest value (kCgGrowth, csrc/kernels.cuh) or p.Ap <= 0.
In a converging solve the rule never fires, so the solve is bit-identical."""
import numpy as np

from oracle import port


def _case():
    L = port.Layout(4, 2, 2)
    A = port.build_A(L).tocsr()
    U, s, _ = np.linalg.svd(A.toarray())
    rank = int((s > s.max() * max(A.shape) * 1e-15).sum())
    return L, A, U[:, rank:]


def test_constraint_rows_are_dependent():
    L, A, null = _case()
    assert null.shape[1] == 73
    assert np.abs(A.T @ null).max() <= 1e-12


def test_plain_cg_diverges_and_the_growth_stop_does_not():
    L, A, null = _case()
    rng = np.random.default_rng(0)
    clean = A @ rng.standard_normal(L.dimx)
    y_clean, _ = port.cg(A, np.zeros(A.shape[0]), clean, 1e-9, 2000)
    rhs = clean + 1e-8 * null @ rng.standard_normal(null.shape[1])
    y_plain, it_plain = port.cg(A, np.zeros(A.shape[0]), rhs, 1e-9, 2000)
    y_stop, it_stop = port.cg(A, np.zeros(A.shape[0]), rhs, 1e-9, 2000, growth_stop=1e4)
    assert it_plain == 2000 and np.linalg.norm(y_plain) > 1e6 * np.linalg.norm(y_clean)
    assert it_stop < 200 and np.linalg.norm(y_stop) <= 2 * np.linalg.norm(y_clean)
    ref = A.T @ y_clean
    assert np.linalg.norm(A.T @ y_stop - ref) <= 1e-5 * np.linalg.norm(ref)


def test_growth_stop_never_fires_in_a_converging_solve():
    from v2rdm_casscf_b200.hamiltonian import synthetic

    a = synthetic(4, 0)
    L = port.Layout(4, a.na, a.nb)
    A = port.build_A(L)
    b = port.build_b(L, A.shape[0])
    c = port.build_c(L, a.h, a.eri())
    runs = []
    for stop in (None, 1e4):
        x, y, z = port.random_guess(L.dimx, A.shape[0])
        runs.append(port.solve(L, A, b, c, x, y, z, 1e-6, 1e-7, cg_growth_stop=stop))
    assert runs[0]["oiter"] == runs[1]["oiter"] and runs[0]["iiter"] == runs[1]["iiter"]
    assert runs[0]["e_primal"] == runs[1]["e_primal"]
