"""Known-answer pin that does not depend on the reference: for two electrons
the D condition is exact, so the D-only boundary-point solve must equal the
singlet full-CI energy (computed densely in tests/helpers.py).  Checked here
for the compiled reference; the GPU solver has the same check in
test_gpu_parity.py."""
import os

import pytest

from tests.helpers import fci_two_electron_singlet


@pytest.mark.parametrize("n,seed", [(3, 0), (4, 1)])
def test_reference_two_electron_d_equals_fci(ref, n, seed):
    from v2rdm_casscf_b200.hamiltonian import synthetic

    a = synthetic(n, seed, electrons=2)
    r = ref.RefSolver([n], [1], positivity="D", r_convergence=1e-7, e_convergence=1e-8)
    r.set_integrals(a.oei_packed, a.qmo, a.nq)
    r.guess()
    r.build_constraints()
    out = r.solve()
    assert out["converged"]
    assert abs(out["e_primal"] + a.enuc - fci_two_electron_singlet(a)) <= 1e-6


def test_reference_three_electron_d_d3_equals_fci(ref):
    # D plus the D3 condition is exact for three electrons (the reference's own
    # H3 test relies on this): the doublet full-CI energy, independent of the
    # reference, must be met
    from tests.helpers import fci_spin_state
    from v2rdm_casscf_b200.hamiltonian import synthetic

    a = synthetic(4, 1, electrons=3)
    r = ref.RefSolver([4], [1], soccpi=[1], multiplicity=2, positivity="D", constrain_d3=True,
                      r_convergence=1e-7, e_convergence=1e-8)
    r.set_integrals(a.oei_packed, a.qmo, a.nq)
    r.guess()
    r.build_constraints()
    out = r.solve()
    assert out["converged"]
    assert abs(out["e_primal"] + a.enuc - fci_spin_state(a, 2)) <= 1e-6


def test_generic_fci_agrees_with_two_electron_formula():
    from tests.helpers import fci_spin_state
    from v2rdm_casscf_b200.hamiltonian import synthetic

    a = synthetic(4, 1, electrons=2)
    assert abs(fci_spin_state(a, 1) - fci_two_electron_singlet(a)) <= 1e-10


def test_reference_four_electron_d_d4_equals_fci(ref):
    # D with the D3 and D4 conditions is exact for four electrons
    from tests.helpers import fci_spin_state
    from v2rdm_casscf_b200.hamiltonian import synthetic

    a = synthetic(4, 1, electrons=4)
    r = ref.RefSolver([4], [2], positivity="D", constrain_d4=True, r_convergence=1e-7, e_convergence=1e-8)
    r.set_integrals(a.oei_packed, a.qmo, a.nq)
    r.guess()
    r.build_constraints()
    out = r.solve()
    assert out["converged"]
    assert abs(out["e_primal"] + a.enuc - fci_spin_state(a, 1)) <= 1e-6


def test_reference_from_least_norm_start_reaches_same_energy(ref):
    # the feasible warm start, applied to the reference's own solver: x0 = A^T w
    # with A A^T w = b, zero duals, mu = 1 reaches the random start's energy
    import numpy as np
    import scipy.sparse.linalg as sla

    from tests.helpers import GOLDEN, load
    from v2rdm_casscf_b200.hamiltonian import synthetic

    g = load(os.path.join(GOLDEN, "solve_synthetic_n4_s0.npz"))
    a = synthetic(4, 0)
    r = ref.RefSolver([4], [a.nb], positivity="DQG", r_convergence=1e-6, e_convergence=1e-7)
    r.set_integrals(a.oei_packed, a.qmo, a.nq)
    r.build_constraints()
    A = _reference_matrix(r)
    b = r.get("b")
    x0 = sla.lsqr(A, b, atol=1e-14, btol=1e-14, iter_lim=20000)[0]
    assert np.linalg.norm(A @ x0 - b) <= 1e-9 * np.linalg.norm(b)
    r.set("x", x0)
    r.set("y", np.zeros(r.ncon))
    r.set("z", np.zeros(r.dimx))
    out = r.solve(mu=1.0)
    assert out["converged"]
    assert abs(out["e_primal"] - float(g["e_primal"])) <= 1e-6
    assert out["oiter"] < int(g["oiter"])  # 780 from the random start


def _reference_matrix(r):
    """A of the reference, column by column through its own bpsdp_Au."""
    import numpy as np
    import scipy.sparse as sp

    A = np.zeros((r.ncon, r.dimx))
    e = np.zeros(r.dimx)
    for j in range(r.dimx):
        e[j] = 1.0
        A[:, j] = r.Au(e)
        e[j] = 0.0
    return sp.csr_matrix(A)
