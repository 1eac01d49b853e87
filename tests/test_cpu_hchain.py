"""Input preparation for the hydrogen-chain workloads (STO-3G integrals, RHF,
Cholesky three-index integrals), checked against the textbook H2 values
(Szabo and Ostlund, Modern Quantum Chemistry, section 3.5.2: R = 1.4 bohr)."""
import numpy as np

from v2rdm_casscf_b200.hchain import ao_integrals, hydrogen_chain, nuclear_repulsion, pivoted_cholesky, rhf


def test_h2_sto3g_integrals_and_rhf():
    c = np.array([[0.0, 0.0, 0.0], [0.0, 0.0, 1.4]])
    S, T, V, eri = ao_integrals(c)
    assert abs(S[0, 1] - 0.6593) < 1e-4
    assert abs(T[0, 0] - 0.7600) < 1e-4 and abs(T[0, 1] - 0.2365) < 1e-4
    assert abs(eri[0, 0, 0, 0] - 0.7746) < 1e-4
    assert abs(eri[0, 0, 1, 1] - 0.5697) < 1e-4
    assert abs(eri[0, 1, 0, 1] - 0.2970) < 1e-4
    assert abs(eri[0, 0, 0, 1] - 0.4441) < 1e-4
    E, C, eps = rhf(S, T + V, eri, 1)
    assert abs(E + nuclear_repulsion(c) - (-1.1167)) < 1e-4
    assert abs(eps[0] - (-0.578)) < 1e-3 and abs(eps[1] - 0.670) < 1e-3


def test_eri_symmetry_and_cholesky():
    c = np.array([[0.0, 0.0, 0.0], [0.0, 0.0, 1.6], [0.0, 0.3, 3.5], [0.2, 0.0, 5.0]])
    _, _, _, eri = ao_integrals(c)
    for perm in ("qprs", "pqsr", "rspq"):
        assert np.allclose(eri, np.einsum("pqrs->" + perm, eri), atol=1e-14)
    n = len(c)
    L = pivoted_cholesky(eri.reshape(n * n, n * n), 1e-12)
    assert np.abs(L.T @ L - eri.reshape(n * n, n * n)).max() < 1e-10


def test_h10_chain_active_space():
    a = hydrogen_chain(10, 0.9)
    assert a.n == 10 and a.na == 5 and a.nb == 5
    # the RHF energy recomputed from the MO integrals and the CD vectors
    g = a.eri()
    occ = range(5)
    e = a.enuc + sum(2 * a.h[i, i] for i in occ) + sum(2 * g[i, i, j, j] - g[i, j, j, i] for i in occ for j in occ)
    assert abs(e - a.scf_energy) < 1e-8


def test_dissociation_scan_converges_along_the_curve():
    from v2rdm_casscf_b200.hchain import hydrogen_scan

    scan = hydrogen_scan(6, 0.6, 3.0, 9)
    e = [a.scf_energy for a in scan]
    k = int(np.argmin(e))
    assert 0 < k < len(e) - 1  # a minimum inside the range
    assert all(e[i] < e[i + 1] for i in range(k, len(e) - 1))  # rising towards dissociation
