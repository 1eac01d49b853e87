"""Linear hydrogen chains in the STO-3G basis: integrals, closed-shell RHF and
Cholesky-decomposed three-index integrals, giving the active-space inputs
(h, L) of the H_n workloads (all orbitals active, no frozen core).

This replaces Psi4's SCF step of the reference workflow for these inputs, so it
is host-side input preparation, not part of the solver.  Only 1s functions
occur, so every integral reduces to the Boys function F0.

Basis: STO-3G for hydrogen (Hehre, Stewart and Pople, J. Chem. Phys. 51, 2657
(1969); zeta = 1.24), exponents and contraction coefficients of the published
set.  Integral formulas for s-type Gaussians as in Szabo and Ostlund, Modern
Quantum Chemistry, appendix A.  The two-electron integrals are decomposed by a
pivoted Cholesky decomposition (the reference's SCF_TYPE CD path gives the
same three-index layout, tei.cc:321), so (pq|rs) = sum_Q L^Q_pq L^Q_rs to the
stated tolerance.
"""
import math

import numpy as np
from scipy.special import erf

from .hamiltonian import ActiveSpace

ANGSTROM_TO_BOHR = 1.0 / 0.529177210903
STO3G_H_EXPONENTS = np.array([3.42525091, 0.62391373, 0.16885540])
STO3G_H_COEFFS = np.array([0.15432897, 0.53532814, 0.44463454])


def _boys0(t):
    t = np.asarray(t, dtype=np.float64)
    out = np.empty_like(t)
    small = t < 1e-12
    out[small] = 1.0 - t[small] / 3.0
    ts = t[~small]
    out[~small] = 0.5 * np.sqrt(np.pi / ts) * erf(np.sqrt(ts))
    return out


def chain_geometry(natoms, spacing_angstrom):
    """Nuclear positions (bohr) of a linear chain along z."""
    z = np.arange(natoms) * spacing_angstrom * ANGSTROM_TO_BOHR
    return np.stack([np.zeros(natoms), np.zeros(natoms), z], axis=1)


def ao_integrals(coords):
    """S, T, V (nao x nao) and (pq|rs) (nao^4) for one STO-3G 1s per H atom."""
    n = len(coords)
    a = STO3G_H_EXPONENTS
    d = STO3G_H_COEFFS * (2.0 * a / np.pi) ** 0.75  # normalised primitives
    # primitive pair quantities for every AO pair (p, q) and primitive pair (i, j)
    A = coords[:, None, None, None, :]
    B = coords[None, :, None, None, :]
    ai = a[None, None, :, None]
    bj = a[None, None, None, :]
    p = (ai + bj) * np.ones((n, n, 1, 1))
    mu = ai * bj / p
    AB2 = np.sum((A - B) ** 2, axis=-1)
    P = (ai[..., None] * A + bj[..., None] * B) / p[..., None]  # (n, n, 3, 3, 3)
    K = np.exp(-mu * AB2)
    dd = d[None, None, :, None] * d[None, None, None, :]
    S = np.sum(dd * (np.pi / p) ** 1.5 * K, axis=(2, 3))
    T = np.sum(dd * mu * (3.0 - 2.0 * mu * AB2) * (np.pi / p) ** 1.5 * K, axis=(2, 3))
    V = np.zeros((n, n))
    for c in coords:
        PC2 = np.sum((P - c) ** 2, axis=-1)
        V -= np.sum(dd * (2.0 * np.pi / p) * K * _boys0(p * PC2), axis=(2, 3))
    # two-electron integrals over contracted pairs
    npair = n * n * 9
    pp = p.reshape(npair)
    KK = (dd * K).reshape(npair)
    PP = P.reshape(npair, 3)
    eri = np.zeros((n * n, n * n))
    for r in range(n * n):
        sl = slice(r * 9, (r + 1) * 9)
        p1, K1, P1 = pp[sl][:, None], KK[sl][:, None], PP[sl][:, None, :]
        PQ2 = np.sum((P1 - PP[None, :, :]) ** 2, axis=-1)
        q = pp[None, :]
        val = 2.0 * np.pi ** 2.5 / (p1 * q * np.sqrt(p1 + q)) * K1 * KK[None, :] * _boys0(p1 * q / (p1 + q) * PQ2)
        eri[r] = val.reshape(9, n * n, 9).sum(axis=(0, 2))
    return S, T, V, eri.reshape(n, n, n, n)


def nuclear_repulsion(coords):
    e = 0.0
    for i in range(len(coords)):
        for j in range(i):
            e += 1.0 / np.linalg.norm(coords[i] - coords[j])
    return e


def rhf(S, Hcore, eri, nocc, max_iter=3000, conv=1e-10, guess=None, damping=0.7):
    """Closed-shell RHF; returns (energy without enuc, C, orbital energies).

    While the orbital gradient is large the density is damped (the Fock
    matrix is built from damping * D_old + (1 - damping) * D_new); close to
    convergence DIIS on the gradient commutator takes over.  guess: starting MO
    coefficients (e.g. from a neighbouring geometry).  Raises if the
    commutator does not fall below 1e-8."""
    s, U = np.linalg.eigh(S)
    X = U @ np.diag(s ** -0.5) @ U.T
    if guess is None:
        e, Cp = np.linalg.eigh(X.T @ Hcore @ X)
        C = X @ Cp
    else:
        C = guess
    D = C[:, :nocc] @ C[:, :nocc].T
    focks, errs = [], []
    E_old = 0.0
    converged = False
    for _ in range(max_iter):
        J = np.einsum("pqrs,rs->pq", eri, D)
        Kx = np.einsum("prqs,rs->pq", eri, D)
        F = Hcore + 2.0 * J - Kx
        E = float(np.sum(D * (Hcore + F)))
        err = X.T @ (F @ D @ S - S @ D @ F) @ X
        gnorm = np.abs(err).max()
        if abs(E - E_old) < conv and gnorm < 1e-9:
            converged = True
            break
        E_old = E
        Fx = F
        if gnorm < 1e-2:
            focks.append(F)
            errs.append(err)
            if len(focks) > 8:
                focks.pop(0)
                errs.pop(0)
            m = len(focks)
            if m > 1:
                Bm = -np.ones((m + 1, m + 1))
                Bm[m, m] = 0.0
                for i in range(m):
                    for j in range(m):
                        Bm[i, j] = np.sum(errs[i] * errs[j])
                rhs = np.zeros(m + 1)
                rhs[m] = -1.0
                try:
                    cvec = np.linalg.solve(Bm, rhs)[:m]
                    Fx = sum(ci * Fi for ci, Fi in zip(cvec, focks))
                except np.linalg.LinAlgError:
                    pass
        e, Cp = np.linalg.eigh(X.T @ Fx @ X)
        C = X @ Cp
        Dn = C[:, :nocc] @ C[:, :nocc].T
        D = Dn if gnorm < 1e-2 else damping * D + (1.0 - damping) * Dn
    if not converged:
        raise RuntimeError("RHF did not converge")
    return E, C, e


def pivoted_cholesky(M, tol):
    """Vectors L (nvec, N) with M ~= L^T L, pivoting on the largest remaining diagonal."""
    N = M.shape[0]
    diag = np.diag(M).copy()
    vecs = []
    while True:
        k = int(np.argmax(diag))
        if diag[k] <= tol:
            break
        col = M[:, k].copy()
        for v in vecs:
            col -= v * v[k]
        v = col / math.sqrt(diag[k])
        vecs.append(v)
        diag -= v * v
        diag[k] = 0.0
        if len(vecs) == N:
            break
    return np.array(vecs)


def hydrogen_chain(natoms, spacing_angstrom, cd_tolerance=1e-10, guess=None):
    """ActiveSpace of an H_natoms chain: all RHF orbitals active, N = natoms (singlet).

    guess: RHF MO coefficients to start from (a neighbouring geometry's)."""
    if natoms % 2:
        raise ValueError("closed-shell chains only (even natoms)")
    coords = chain_geometry(natoms, spacing_angstrom)
    S, T, V, eri = ao_integrals(coords)
    Hc = T + V
    enuc = nuclear_repulsion(coords)
    E, C, eps = rhf(S, Hc, eri, natoms // 2, guess=guess)
    n = natoms
    Lao = pivoted_cholesky(eri.reshape(n * n, n * n), cd_tolerance).reshape(-1, n, n)
    Lmo = np.einsum("pi,Qpq,qj->Qij", C, Lao, C)
    Lmo = 0.5 * (Lmo + Lmo.transpose(0, 2, 1))
    h = C.T @ Hc @ C
    h = 0.5 * (h + h.T)
    a = ActiveSpace(h, Lmo, natoms // 2, natoms // 2, enuc=enuc, name=f"H{natoms} chain {spacing_angstrom} A STO-3G")
    a.scf_energy = E + enuc
    a.orbital_energies = eps
    a.mo_coefficients = C
    return a


def hydrogen_scan(natoms=20, first=0.6, last=3.0, points=64):
    """The symmetric dissociation scan: spacings linear in [first, last] Angstrom,
    each RHF started from the previous geometry's orbitals."""
    out, guess = [], None
    for r in np.linspace(first, last, points):
        a = hydrogen_chain(natoms, float(r), guess=guess)
        guess = a.mo_coefficients
        out.append(a)
    return out
