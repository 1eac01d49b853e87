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
