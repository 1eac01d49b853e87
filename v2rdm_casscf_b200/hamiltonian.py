"""Active-space Hamiltonians in the layout the v2RDM plugin consumes.

The plugin receives one-electron integrals packed per irrep as a lower
triangle (``oei_full_sym_``, v2rdm_solver.cc / tei.cc:130) and three-index
integrals ``Qmo[Q * ntri + INDEX(p, q)]`` with ``ntri = nmo (nmo + 1) / 2``
(tei.cc:321).  This module builds such inputs for the workloads the solver is
measured on:

* ``synthetic(n, seed)``: the seeded active space of the batched workload
  (singlet; N = n electrons, N = n - 1 for odd n).
  h is symmetric with diagonal ~ U(-2.0, -0.5) Eh and off-diagonal
  ~ N(0, 0.1^2); g_pqrs = sum_Q L^Q_pq L^Q_rs with 3n symmetric Cholesky
  vectors whose entries are ~ N(0, 0.25^2), so the ERI tensor is PSD with
  8-fold symmetry.  Random numbers come from numpy's Philox4x32-10
  counter-based generator keyed by (seed, stream), so instance s is the same
  on every machine independently of how many instances are generated.
"""
import numpy as np


def tri(n):
    return n * (n + 1) // 2


def pack_lower(m):
    """Row-major packed lower triangle: element (i, j), i >= j, at i(i+1)/2 + j."""
    n = m.shape[0]
    i, j = np.tril_indices(n)
    out = np.zeros(tri(n))
    out[i * (i + 1) // 2 + j] = m[i, j]
    return out


def unpack_lower(p, n):
    m = np.zeros((n, n))
    i, j = np.tril_indices(n)
    m[i, j] = p[i * (i + 1) // 2 + j]
    m[j, i] = p[i * (i + 1) // 2 + j]
    return m


class ActiveSpace:
    """Integrals for an all-active C1 space of n orbitals with N = na + nb electrons."""

    def __init__(self, h, L, na, nb, enuc=0.0, name=""):
        self.h = np.asarray(h, dtype=np.float64)
        self.L = np.asarray(L, dtype=np.float64)  # (nQ, n, n), each symmetric
        self.n = self.h.shape[0]
        self.nq = self.L.shape[0]
        self.na = int(na)
        self.nb = int(nb)
        self.enuc = float(enuc)
        self.name = name

    @property
    def oei_packed(self):
        return pack_lower(self.h)

    @property
    def qmo(self):
        """(nQ, ntri) three-index integrals, flattened Q-major as the plugin stores them."""
        return np.stack([pack_lower(l) for l in self.L]).reshape(-1)

    def eri(self):
        """(pq|rs) as a dense n^4 array (small n only)."""
        return np.einsum("Qpq,Qrs->pqrs", self.L, self.L)

    @property
    def doccpi(self):
        return [self.nb]

    @property
    def soccpi(self):
        return [self.na - self.nb]

    @property
    def multiplicity(self):
        return self.na - self.nb + 1


def synthetic(n, seed, nq=None, electrons=None):
    """Seeded synthetic singlet active space of n orbitals.

    The batched workload asks for N = n electrons in a singlet; an odd n cannot
    hold a singlet with n electrons, so odd n get N = n - 1 (still a singlet,
    half filling rounded down).  ``electrons`` overrides N (high-spin for odd N).
    """
    nq = 3 * n if nq is None else nq
    rng_h = np.random.Generator(np.random.Philox(key=[seed, 0]))
    rng_l = np.random.Generator(np.random.Philox(key=[seed, 1]))
    h = rng_h.normal(0.0, 0.1, size=(n, n))
    h = np.tril(h, -1)
    h = h + h.T
    h[np.diag_indices(n)] = rng_h.uniform(-2.0, -0.5, size=n)
    L = rng_l.normal(0.0, 0.25, size=(nq, n, n))
    L = np.tril(L)
    L = L + np.transpose(np.tril(L, -1), (0, 2, 1))
    N = (n - n % 2) if electrons is None else int(electrons)
    return ActiveSpace(h, L, N - N // 2, N // 2, 0.0, name=f"synthetic(n={n},seed={seed},N={N})")


def batch_sizes(count=256, nmin=8, nmax=20, seed=2024):
    """Orbital counts of the batched workload: n ~ U{nmin..nmax}, one per instance."""
    rng = np.random.Generator(np.random.Philox(key=[seed, 7]))
    return rng.integers(nmin, nmax + 1, size=count)
