"""ctypes access to the reference BPSDP hot path compiled in oracle/_ref.

TEST INFRASTRUCTURE ONLY: used by tests/, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of bench.py as the checker, never by the product.

``RefSolver`` wraps one ``v2RDMSolver`` of the reference (its layout code from
v2rdm_solver.cc:487-1285, the constraint maps of d2.cc/spin.cc/q2.cc/g2.cc/
t1.cc/t2.cc, RepackIntegrals from tei.cc, Guess/BuildConstraints/Update_xz
from v2rdm_solver.cc:2386-3289 and CGSolver from cg_solver.cc), driven by the
outer loop restated in oracle/ref_harness.cc (v2rdm_solver.cc:1778-1908).
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_ref", "libv2rdm_ref.so")

_lib = None


def available():
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise RuntimeError(f"oracle library missing: {LIB_PATH} (run `make -C oracle`)")
        L = ctypes.CDLL(LIB_PATH)
        P = ctypes.c_void_p
        I = ctypes.c_int
        D = ctypes.c_double
        IP = ctypes.POINTER(ctypes.c_int)
        DP = ctypes.POINTER(ctypes.c_double)
        S = ctypes.c_char_p
        L.oref_create.restype = P
        L.oref_create.argtypes = [I, IP, IP, IP, IP, IP, IP, IP, I, S, I, I, D, D, D, I, I]
        L.oref_last_error.restype = S
        L.oref_destroy.argtypes = [P]
        L.oref_dimx.restype = ctypes.c_long
        L.oref_dimx.argtypes = [P]
        L.oref_ncon.restype = ctypes.c_long
        L.oref_ncon.argtypes = [P]
        L.oref_nblocks.argtypes = [P]
        L.oref_block_dims.argtypes = [P, IP]
        L.oref_offsets.argtypes = [P, S, IP]
        L.oref_counts.argtypes = [P, S, IP]
        L.oref_ibas.argtypes = [P, S, I, IP]
        L.oref_set_integrals.argtypes = [P, DP, DP, I, D]
        L.oref_efzc.restype = D
        L.oref_efzc.argtypes = [P]
        L.oref_get.argtypes = [P, S, DP]
        L.oref_set.argtypes = [P, S, DP]
        L.oref_guess.argtypes = [P]
        L.oref_build_constraints.argtypes = [P]
        L.oref_Au.argtypes = [P, DP, DP]
        L.oref_ATu.argtypes = [P, DP, DP]
        L.oref_update_xz.argtypes = [P, D]
        L.oref_solve.argtypes = [P, D, D, I, I, DP, DP, I]
        L.oref_set_threads.argtypes = [I]
        L.oref_set_next_energies.argtypes = [DP, I]
        L.oref_set_next_spin_adapt.argtypes = [I, I, I, I]
        L.oref_spatial_dims.restype = ctypes.c_long
        L.oref_spatial_dims.argtypes = [P, ctypes.POINTER(ctypes.c_long), ctypes.POINTER(ctypes.c_long)]
        L.oref_pack_spatial.argtypes = [P, DP, DP]
        _lib = L
    return _lib


def _iarr(a):
    a = np.ascontiguousarray(a, dtype=np.int32)
    return a, a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


def _dptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def set_threads(n):
    lib().oref_set_threads(int(n))


class RefSolver:
    """One reference solver instance.

    Orbital counts are per irrep, like Psi4's Dimension objects.  Options
    mirror the plugin's (plugin.cc:66-124).
    """

    def __init__(self, nmopi, doccpi, soccpi=None, frzcpi=None, rstcpi=None, rstvpi=None, frzvpi=None,
                 multiplicity=1, positivity="DQG", constrain_spin=True, constrain_sz=True,
                 r_convergence=1e-4, e_convergence=1e-4, cg_convergence=1e-9, maxiter=10000,
                 cg_maxiter=10000, energies=None, spin_adapt_q2=False, spin_adapt_g2=False,
                 constrain_d3=False, constrain_d4=False):
        nirrep = len(nmopi)
        lib().oref_set_next_spin_adapt(int(bool(spin_adapt_q2)), int(bool(spin_adapt_g2)), int(bool(constrain_d3)),
                                       int(bool(constrain_d4)))
        if energies is not None:  # orbital energies, all orbitals in Pitzer order
            e = np.ascontiguousarray(energies, dtype=np.float64)
            lib().oref_set_next_energies(_dptr(e), int(e.size))
        z = [0] * nirrep
        arrs = [_iarr(v if v is not None else z) for v in
                (nmopi, frzcpi, rstcpi, rstvpi, frzvpi, doccpi, soccpi)]
        self._keep = arrs
        L = lib()
        self.h = L.oref_create(nirrep, *[p for _, p in arrs], int(multiplicity), positivity.encode(),
                               int(constrain_spin), int(constrain_sz), float(r_convergence),
                               float(e_convergence), float(cg_convergence), int(maxiter), int(cg_maxiter))
        if not self.h:
            raise RuntimeError("oracle setup failed: " + L.oref_last_error().decode())
        self.nirrep = nirrep
        self.dimx = L.oref_dimx(self.h)
        self.ncon = L.oref_ncon(self.h)
        nb = L.oref_nblocks(self.h)
        dims, p = _iarr(np.zeros(nb))
        L.oref_block_dims(self.h, p)
        self.block_dims = dims.copy()

    def __del__(self):
        if getattr(self, "h", None):
            lib().oref_destroy(self.h)
            self.h = None

    def offsets(self, family):
        out, p = _iarr(np.zeros(self.nirrep))
        n = lib().oref_offsets(self.h, family.encode(), p)
        return out.copy() if n else None

    def counts(self, what):
        out, p = _iarr(np.zeros(self.nirrep))
        lib().oref_counts(self.h, what.encode(), p)
        return out.copy()

    def ibas(self, what, irrep, amo):
        out, p = _iarr(np.zeros(amo * amo))
        lib().oref_ibas(self.h, what.encode(), irrep, p)
        return out.reshape(amo, amo).copy()

    def set_integrals(self, oei_packed, qmo, nq, enuc=0.0):
        oei = np.ascontiguousarray(oei_packed, dtype=np.float64)
        q = np.ascontiguousarray(qmo, dtype=np.float64)
        if lib().oref_set_integrals(self.h, _dptr(oei), _dptr(q), int(nq), float(enuc)) != 0:
            raise RuntimeError(lib().oref_last_error().decode())

    @property
    def efzc(self):
        return lib().oref_efzc(self.h)

    def get(self, which):
        n = self.ncon if which in ("y", "b") else self.dimx
        out = np.zeros(n)
        if lib().oref_get(self.h, which.encode(), _dptr(out)) != 0:
            raise RuntimeError(lib().oref_last_error().decode())
        return out

    def set(self, which, v):
        n = self.ncon if which in ("y", "b") else self.dimx
        a = np.ascontiguousarray(v, dtype=np.float64)
        assert a.size == n
        lib().oref_set(self.h, which.encode(), _dptr(a))

    def guess(self):
        lib().oref_guess(self.h)

    def build_constraints(self):
        lib().oref_build_constraints(self.h)

    def Au(self, u):
        u = np.ascontiguousarray(u, dtype=np.float64)
        assert u.size == self.dimx
        out = np.zeros(self.ncon)
        lib().oref_Au(self.h, _dptr(u), _dptr(out))
        return out

    def ATu(self, u):
        u = np.ascontiguousarray(u, dtype=np.float64)
        assert u.size == self.ncon
        out = np.zeros(self.dimx)
        lib().oref_ATu(self.h, _dptr(u), _dptr(out))
        return out

    def update_xz(self, mu):
        lib().oref_update_xz(self.h, float(mu))

    def pack_spatial_density(self):
        """(d1, d2) of PackSpatialDensity for the current x (v2rdm_solver.cc:3664-3773)."""
        n1, n2 = ctypes.c_long(), ctypes.c_long()
        lib().oref_spatial_dims(self.h, ctypes.byref(n1), ctypes.byref(n2))
        d1, d2 = np.zeros(n1.value), np.zeros(n2.value)
        lib().oref_pack_spatial(self.h, _dptr(d1), _dptr(d2))
        return d1, d2

    def solve(self, tau=1.0, mu=1.0, mu_update_frequency=500, max_outer=0, trace_cap=0):
        res = np.zeros(16)
        trace = np.zeros(8 * max(trace_cap, 1))
        st = lib().oref_solve(self.h, float(tau), float(mu), int(mu_update_frequency), int(max_outer),
                              _dptr(res), _dptr(trace), int(trace_cap))
        if st < 0:
            raise RuntimeError(lib().oref_last_error().decode())
        out = dict(converged=(st == 0), e_primal=res[0], e_dual=res[1], ep=res[2], ed=res[3], mu=res[4],
                   oiter=int(res[5]), iiter=int(res[6]), t_cg=res[7], t_xz=res[8], t_total=res[9],
                   efzc=res[10])
        if trace_cap:
            n = min(out["oiter"], trace_cap)
            out["trace"] = trace[: 8 * n].reshape(n, 8).copy()
        return out
