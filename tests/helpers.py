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
