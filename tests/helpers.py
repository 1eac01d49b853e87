import os

import numpy as np
import scipy.sparse as sp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def load(path):
    return dict(np.load(path, allow_pickle=False))


def make_solver(V, g, **kw):
    """Product solver for a maps_*.npz golden case."""
    docc, socc = g["doccpi"], g["soccpi"]
    na, nb = int(docc.sum() + socc.sum()), int(docc.sum())
    opts = dict(POSITIVITY=str(g["positivity"]), CONSTRAIN_SPIN=bool(g["constrain_spin"]),
                CONSTRAIN_SZ=bool(g["constrain_sz"]))
    if "spin_adapt_q2" in g:
        opts.update(SPIN_ADAPT_Q2=bool(g["spin_adapt_q2"]), SPIN_ADAPT_G2=bool(g["spin_adapt_g2"]))
    if "constrain_d3" in g:
        opts.update(CONSTRAIN_D3=bool(g["constrain_d3"]))
    if "constrain_d4" in g:
        opts.update(CONSTRAIN_D4=bool(g["constrain_d4"]))
    return V.V2RDMSolver(g["amopi"].tolist(), na, nb, int(socc.sum()) + 1, options=opts, **kw)


def csr_of(s):
    rp, col, val = s.A_csr()
    return sp.csr_matrix((val, col, rp), shape=(s.nconstraints, s.dimx))


def fci_two_electron_singlet(a):
    """Exact ground-state energy of a two-electron singlet in the active space
    (dense diagonalisation over symmetric spatial pair functions), plus enuc.

    For two electrons the D condition is exact, so a D-only v2RDM solve must
    reach this energy: a check that does not go through the reference."""
    n = a.n
    h, g = a.h, a.eri()
    eye = np.eye(n)
    H = (np.einsum("ik,jl->ijkl", h, eye) + np.einsum("ik,jl->ijkl", eye, h)
         + np.einsum("ikjl->ijkl", g)).reshape(n * n, n * n)
    cols = []
    for i in range(n):
        for j in range(i, n):
            v = np.zeros((n, n))
            v[i, j] += 1.0
            v[j, i] += 1.0
            cols.append(v.ravel() / np.linalg.norm(v))
    Q = np.array(cols).T
    return float(np.linalg.eigvalsh(Q.T @ H @ Q)[0]) + a.enuc


def _apply(det, ops):
    """Apply a product of creation (+p) / annihilation (-p - 1) operators, rightmost
    first, to a determinant given as a bit string over spin orbitals."""
    sign = 1
    for op in reversed(ops):
        p = op if op >= 0 else -op - 1
        occ = (det >> p) & 1
        if (op >= 0) == bool(occ):
            return 0, 0
        if bin(det & ((1 << p) - 1)).count("1") % 2:
            sign = -sign
        det ^= 1 << p
    return sign, det


def fci_spin_state(a, multiplicity):
    """Lowest full-CI energy (plus enuc) of the active space with a.na alpha and
    a.nb beta electrons among the states of the given spin multiplicity; dense,
    for a handful of orbitals.  Spin orbitals: alpha p -> p, beta p -> n + p."""
    from itertools import combinations

    n = a.n
    h, g = a.h, a.eri()
    dets = []
    for al in combinations(range(n), a.na):
        for be in combinations(range(n), a.nb):
            d = 0
            for p in al:
                d |= 1 << p
            for p in be:
                d |= 1 << (n + p)
            dets.append(d)
    index = {d: i for i, d in enumerate(dets)}
    N = len(dets)
    H = np.zeros((N, N))
    S2 = np.zeros((N, N))
    for col, d in enumerate(dets):
        for sp in (0, n):
            for p in range(n):
                for q in range(n):
                    s, e = _apply(d, [sp + p, -(sp + q) - 1])
                    if s and e in index:
                        H[index[e], col] += s * h[p, q]
        for s1 in (0, n):
            for s2 in (0, n):
                for p in range(n):
                    for q in range(n):
                        for r in range(n):
                            for t in range(n):
                                v = g[p, q, r, t]
                                if v == 0.0:
                                    continue
                                s, e = _apply(d, [s1 + p, s2 + r, -(s2 + t) - 1, -(s1 + q) - 1])
                                if s and e in index:
                                    H[index[e], col] += 0.5 * s * v
        # S^2 = S- S+ + Sz (Sz + 1)
        sz = 0.5 * (a.na - a.nb)
        S2[col, col] += sz * (sz + 1.0)
        for p in range(n):
            for q in range(n):
                s, e = _apply(d, [n + p, -p - 1, q, -(n + q) - 1])
                if s and e in index:
                    S2[index[e], col] += s
    w, V = np.linalg.eigh(H)
    spin = 0.5 * (multiplicity - 1)
    s2 = np.einsum("ik,ij,jk->k", V, S2, V)
    ok = np.abs(s2 - spin * (spin + 1.0)) < 1e-6
    return float(w[ok][0]) + a.enuc
