"""Known-answer pin that does not depend on the reference: for two electrons
the D condition is exact, so the D-only boundary-point solve must equal the
singlet full-CI energy (computed densely in tests/helpers.py).  Checked here
for the compiled reference; the GPU solver has the same check in
test_gpu_parity.py."""
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
