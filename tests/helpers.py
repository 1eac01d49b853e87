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
    return V.V2RDMSolver(g["amopi"].tolist(), na, nb, int(socc.sum()) + 1, options=opts, **kw)


def csr_of(s):
    rp, col, val = s.A_csr()
    return sp.csr_matrix((val, col, rp), shape=(s.nconstraints, s.dimx))
