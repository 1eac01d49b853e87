"""B200 boundary-point SDP solver for the active-space hot path of v2RDM-CASSCF.

Python mirror of the plugin surface over the C ABI in include/v2rdm_gpu.h
(libv2rdm_b200.so, built in-tree by ``v2rdm_casscf_b200.build``).  Option names
and defaults follow the plugin's read_options (plugin.cc:66-124); the solver
object follows v2RDMSolver (v2rdm_solver.h:79-575): its primal/dual vectors x,
y, z, the PSD block list ``dimensions``, and ``compute_energy``.

The solve runs on the GPU only.  If the library is missing, importing works but
creating a solver raises; there is no CPU path.
"""
import ctypes
import os

import numpy as np

from . import hamiltonian  # noqa: F401

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libv2rdm_b200.so")

V2G_OK = 0
V2G_ERR_ARG = -1
V2G_ERR_CUDA = -2
V2G_ERR_NOT_CONVERGED = -3
V2G_ERR_NONFINITE = -4
V2G_ERR_UNSUPPORTED = -5
V2G_ERR_NO_DEVICE = -6

# Functions declared in include/v2rdm_gpu.h (checked by the tests).
EXPORTS = [
    "v2g_default_options", "v2g_last_error", "v2g_create", "v2g_destroy", "v2g_dimx", "v2g_nconstraints",
    "v2g_nblocks", "v2g_block_dims", "v2g_set_hamiltonian", "v2g_get_c", "v2g_get_b", "v2g_efzc",
    "v2g_guess_random", "v2g_set_state", "v2g_get_state", "v2g_apply_A", "v2g_apply_AT", "v2g_apply_A_device",
    "v2g_apply_AT_device", "v2g_update_xz", "v2g_solve", "v2g_solve_batch", "v2g_A_nnz", "v2g_export_A",
    "v2g_trace", "v2g_last_batch_stats", "v2g_apply_A_batched_device", "v2g_apply_AT_batched_device",
    "v2g_update_xz_noalloc", "v2g_spatial_density_dims", "v2g_pack_spatial_density", "v2g_block_gemm_device",
    "v2g_time_maps", "v2g_time_block_gemm",
    "v2g_write_checkpoint", "v2g_read_checkpoint", "v2g_set_active_orbital_energies", "v2g_solve_continue",
    "v2g_ws_create", "v2g_ws_destroy", "v2g_ws_num_params", "v2g_ws_get_params", "v2g_ws_set_params", "v2g_ws_rows",
    "v2g_ws_features", "v2g_ws_targets", "v2g_ws_forward", "v2g_ws_gradient", "v2g_ws_train", "v2g_ws_propose",
]


class Options(ctypes.Structure):
    _fields_ = [
        ("positivity", ctypes.c_char_p),
        ("constrain_spin", ctypes.c_int),
        ("constrain_sz", ctypes.c_int),
        ("r_convergence", ctypes.c_double),
        ("e_convergence", ctypes.c_double),
        ("cg_convergence", ctypes.c_double),
        ("maxiter", ctypes.c_int),
        ("cg_maxiter", ctypes.c_int),
        ("tau_parameter", ctypes.c_double),
        ("mu_update_frequency", ctypes.c_int),
        ("device", ctypes.c_int),
        ("record_trace", ctypes.c_int),
        ("profile", ctypes.c_int),
        ("adaptive_projection", ctypes.c_int),
        ("cg_tolerance_factor", ctypes.c_double),
        ("spin_adapt_q2", ctypes.c_int),
        ("spin_adapt_g2", ctypes.c_int),
        ("constrain_d3", ctypes.c_int),
        ("constrain_d4", ctypes.c_int),
        ("start", ctypes.c_int),
        ("cg_extrapolate", ctypes.c_int),
        ("anderson_memory", ctypes.c_int),
        ("mixed_precision", ctypes.c_int),
    ]


class BatchStats(ctypes.Structure):
    _fields_ = [
        ("device_seconds", ctypes.c_double),
        ("e2e_seconds", ctypes.c_double),
        ("kernel_launches", ctypes.c_long),
        ("map_seconds", ctypes.c_double),
        ("map_launches", ctypes.c_long),
        ("map_bytes", ctypes.c_double),
        ("groups", ctypes.c_long),
        ("h2d_bytes", ctypes.c_double),
        ("d2h_bytes", ctypes.c_double),
        ("refine_sweeps", ctypes.c_long),
        ("jacobi_sweeps", ctypes.c_long),
        ("jacobi_blocks", ctypes.c_long),
        ("jacobi_unconverged", ctypes.c_long),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class Result(ctypes.Structure):
    _fields_ = [
        ("e_total", ctypes.c_double),
        ("e_primal", ctypes.c_double),
        ("e_dual", ctypes.c_double),
        ("ep", ctypes.c_double),
        ("ed", ctypes.c_double),
        ("mu", ctypes.c_double),
        ("efzc", ctypes.c_double),
        ("enuc", ctypes.c_double),
        ("oiter", ctypes.c_long),
        ("iiter", ctypes.c_long),
        ("status", ctypes.c_int),
        ("t_cg", ctypes.c_double),
        ("t_xz", ctypes.c_double),
        ("t_total", ctypes.c_double),
        ("cg_stalls", ctypes.c_long),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_lib = None


def lib():
    """The loaded solver library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: run `python -m v2rdm_casscf_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        P, I, D, L_ = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_long
        IP = ctypes.POINTER(ctypes.c_int)
        DP = ctypes.POINTER(ctypes.c_double)
        LP = ctypes.POINTER(ctypes.c_long)
        L.v2g_default_options.argtypes = [ctypes.POINTER(Options)]
        L.v2g_last_error.restype = ctypes.c_char_p
        L.v2g_create.argtypes = [ctypes.POINTER(Options), I, IP, IP, IP, IP, IP, I, I, I, ctypes.POINTER(P)]
        L.v2g_destroy.argtypes = [P]
        for f in ("v2g_dimx", "v2g_nconstraints", "v2g_A_nnz"):
            getattr(L, f).restype = L_
            getattr(L, f).argtypes = [P]
        L.v2g_nblocks.argtypes = [P]
        L.v2g_block_dims.argtypes = [P, IP]
        L.v2g_set_hamiltonian.argtypes = [P, DP, DP, I, D]
        L.v2g_get_c.argtypes = [P, DP]
        L.v2g_get_b.argtypes = [P, DP]
        L.v2g_efzc.restype = D
        L.v2g_efzc.argtypes = [P]
        L.v2g_guess_random.argtypes = [P]
        L.v2g_set_state.argtypes = [P, DP, DP, DP, D]
        L.v2g_get_state.argtypes = [P, DP, DP, DP, DP]
        for f in ("v2g_apply_A", "v2g_apply_AT"):
            getattr(L, f).argtypes = [P, DP, DP]
        for f in ("v2g_apply_A_device", "v2g_apply_AT_device"):
            getattr(L, f).argtypes = [P, P, P]
        L.v2g_update_xz.argtypes = [P, D]
        L.v2g_update_xz_noalloc.argtypes = [P, D, P, P, P, P, P]
        L.v2g_spatial_density_dims.argtypes = [P, LP, LP]
        L.v2g_pack_spatial_density.argtypes = [P, DP, DP, DP]
        L.v2g_write_checkpoint.argtypes = [P, ctypes.c_char_p]
        L.v2g_set_active_orbital_energies.argtypes = [P, DP]
        L.v2g_read_checkpoint.argtypes = [P, ctypes.c_char_p]
        L.v2g_solve.argtypes = [P, ctypes.POINTER(Result)]
        L.v2g_solve_continue.argtypes = [P, I, ctypes.POINTER(Result)]
        L.v2g_solve_batch.argtypes = [ctypes.POINTER(P), I, ctypes.POINTER(Result)]
        L.v2g_export_A.argtypes = [P, LP, IP, DP]
        L.v2g_trace.restype = L_
        L.v2g_trace.argtypes = [P, DP, L_]
        L.v2g_last_batch_stats.argtypes = [ctypes.POINTER(BatchStats)]
        for f in ("v2g_apply_A_batched_device", "v2g_apply_AT_batched_device"):
            getattr(L, f).argtypes = [P, I, P, P, P]
        L.v2g_block_gemm_device.argtypes = [I, IP, P, I, P, I, P, P, I, I]
        L.v2g_time_maps.argtypes = [P, I, I, DP, DP]
        L.v2g_time_block_gemm.argtypes = [I, IP, P, P, P, I, I, I, DP]
        FP = ctypes.POINTER(ctypes.c_float)
        L.v2g_ws_create.argtypes = [I, I, ctypes.c_ulonglong, ctypes.POINTER(P)]
        L.v2g_ws_destroy.argtypes = [P]
        L.v2g_ws_num_params.restype = L_
        L.v2g_ws_num_params.argtypes = [P]
        L.v2g_ws_get_params.argtypes = [P, FP]
        L.v2g_ws_set_params.argtypes = [P, FP]
        L.v2g_ws_rows.restype = L_
        L.v2g_ws_rows.argtypes = [P]
        L.v2g_ws_features.argtypes = [P, FP]
        L.v2g_ws_targets.argtypes = [P, FP]
        L.v2g_ws_forward.argtypes = [P, L_, FP, FP]
        L.v2g_ws_gradient.argtypes = [P, L_, FP, FP, DP, FP]
        L.v2g_ws_train.argtypes = [P, L_, FP, FP, I, I, ctypes.c_float, DP]
        L.v2g_ws_propose.argtypes = [P, P, I]
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _ip(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


class V2GError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"v2g error {code}: {msg}")
        self.code = code


def _check(code):
    if code != V2G_OK:
        raise V2GError(code, lib().v2g_last_error().decode())


# Plugin options on this path and their defaults (plugin.cc:66-124).
DEFAULT_OPTIONS = dict(
    POSITIVITY="DQG",
    CONSTRAIN_SPIN=True,
    CONSTRAIN_SZ=True,
    R_CONVERGENCE=1e-4,
    E_CONVERGENCE=1e-4,
    CG_CONVERGENCE=1e-9,
    MAXITER=10000,
    CG_MAXITER=10000,
    TAU_PARAMETER=1.0,
    MU_UPDATE_FREQUENCY=500,
    SPIN_ADAPT_Q2=False,
    SPIN_ADAPT_G2=False,
    CONSTRAIN_D3=False,
    CONSTRAIN_D4=False,
)


class V2RDMSolver:
    """One active-space BPSDP problem on the GPU.

    Parameters mirror Psi4's per-irrep orbital arrays (FROZEN_DOCC,
    RESTRICTED_DOCC, ACTIVE, RESTRICTED_UOCC, FROZEN_UOCC) and the reference
    wavefunction's nalpha/nbeta/multiplicity; ``options`` takes the plugin's
    option names.  ``projection="adaptive"`` lets Update_xz accept an
    eigendecomposition whose residual is below 0.01 min(eps(p), eps(d)) (the
    CG tolerance rule); the default "exact" converges every projection, as
    the plugin does.  ``cg_tolerance_factor`` replaces the 0.01 of the CG
    tolerance rule 0.01 min(eps(p), eps(d)).  ``cg_extrapolate=True`` starts
    each outer iteration's CG from y_k + (y_k - y_{k-1}) instead of y_k (same
    stopping test, fewer CG iterations).  ``anderson_memory=m`` (1..16)
    accelerates the outer iteration on (x, z) with the last m step
    differences (Anderson's method; the stopping test and energies are those
    of the plain step).  ``mixed_precision=True`` (with the adaptive
    projection) runs the dense products of the large blocks' projection on
    the tensor cores (3xTF32, FP32 accuracy) while the projection tolerance is
    at least 1e-5, and in FP64 after that.
    """

    def __init__(self, active, nalpha, nbeta, multiplicity=1, frozen_docc=None, restricted_docc=None,
                 restricted_uocc=None, frozen_uocc=None, options=None, device=0, record_trace=False,
                 profile=False, projection="exact", cg_tolerance_factor=0.01, start="state",
                 cg_extrapolate=False, anderson_memory=0, mixed_precision=False):
        L = lib()
        self.active = list(active)
        opts = dict(DEFAULT_OPTIONS)
        for k, v in (options or {}).items():
            k = k.upper()
            if k not in opts:
                raise KeyError(f"unknown option {k}")
            opts[k] = v
        self.options = opts
        o = Options()
        L.v2g_default_options(ctypes.byref(o))
        self._pos = str(opts["POSITIVITY"]).upper().encode()
        o.positivity = self._pos
        o.constrain_spin = int(bool(opts["CONSTRAIN_SPIN"]))
        o.constrain_sz = int(bool(opts["CONSTRAIN_SZ"]))
        o.r_convergence = float(opts["R_CONVERGENCE"])
        o.e_convergence = float(opts["E_CONVERGENCE"])
        o.cg_convergence = float(opts["CG_CONVERGENCE"])
        o.maxiter = int(opts["MAXITER"])
        o.cg_maxiter = int(opts["CG_MAXITER"])
        o.tau_parameter = float(opts["TAU_PARAMETER"])
        o.mu_update_frequency = int(opts["MU_UPDATE_FREQUENCY"])
        o.device = int(device)
        o.record_trace = int(bool(record_trace))
        o.profile = int(bool(profile))
        if projection not in ("exact", "adaptive"):
            raise ValueError("projection is 'exact' or 'adaptive'")
        o.adaptive_projection = int(projection == "adaptive")
        o.cg_tolerance_factor = float(cg_tolerance_factor)
        o.spin_adapt_q2 = int(bool(opts["SPIN_ADAPT_Q2"]))
        o.spin_adapt_g2 = int(bool(opts["SPIN_ADAPT_G2"]))
        o.constrain_d3 = int(bool(opts["CONSTRAIN_D3"]))
        o.constrain_d4 = int(bool(opts["CONSTRAIN_D4"]))
        if start not in ("state", "feasible", "learned"):
            raise ValueError("start is 'state' (guess()/set_state), 'feasible' or 'learned'")
        o.start = {"state": 0, "feasible": 1, "learned": 2}[start]
        o.cg_extrapolate = int(bool(cg_extrapolate))
        o.anderson_memory = int(anderson_memory)
        o.mixed_precision = int(bool(mixed_precision))
        nirrep = len(active)
        zero = [0] * nirrep
        arrs = [np.ascontiguousarray(v if v is not None else zero, dtype=np.int32)
                for v in (frozen_docc, restricted_docc, active, restricted_uocc, frozen_uocc)]
        self.spaces = arrs
        h = ctypes.c_void_p()
        _check(L.v2g_create(ctypes.byref(o), nirrep, *[_ip(a) for a in arrs], int(nalpha), int(nbeta),
                            int(multiplicity), ctypes.byref(h)))
        self.h = h
        self.nirrep = nirrep
        self.dimx = L.v2g_dimx(h)
        self.nconstraints = L.v2g_nconstraints(h)
        nb = L.v2g_nblocks(h)
        dims = np.zeros(nb, dtype=np.int32)
        L.v2g_block_dims(h, _ip(dims))
        self.dimensions = dims
        self.result = None

    def __del__(self):
        h = getattr(self, "h", None)
        if h is not None and h.value and _lib is not None:
            try:
                _lib.v2g_destroy(h)
            except Exception:
                pass
            self.h = None

    # -- inputs ---------------------------------------------------------------
    def set_hamiltonian(self, oei_packed, qmo, nq, enuc=0.0):
        oei = np.ascontiguousarray(oei_packed, dtype=np.float64)
        q = np.ascontiguousarray(qmo, dtype=np.float64)
        _check(lib().v2g_set_hamiltonian(self.h, _dp(oei), _dp(q), int(nq), float(enuc)))

    @classmethod
    def from_active_space(cls, space, options=None, **kw):
        """Solver for a hamiltonian.ActiveSpace (all orbitals active, C1)."""
        s = cls([space.n], space.na, space.nb, space.multiplicity, options=options, **kw)
        s.set_hamiltonian(space.oei_packed, space.qmo, space.nq, space.enuc)
        return s

    @property
    def c(self):
        out = np.zeros(self.dimx)
        _check(lib().v2g_get_c(self.h, _dp(out)))
        return out

    @property
    def b(self):
        out = np.zeros(self.nconstraints)
        _check(lib().v2g_get_b(self.h, _dp(out)))
        return out

    @property
    def efzc(self):
        return lib().v2g_efzc(self.h)

    def guess(self):
        """The plugin's TPDM_GUESS=RANDOM start (srand(0))."""
        _check(lib().v2g_guess_random(self.h))

    def set_state(self, x, y, z, mu=1.0):
        x, y, z = (np.ascontiguousarray(v, dtype=np.float64) for v in (x, y, z))
        assert x.size == self.dimx and z.size == self.dimx and y.size == self.nconstraints
        _check(lib().v2g_set_state(self.h, _dp(x), _dp(y), _dp(z), float(mu)))

    def get_state(self):
        x, z = np.zeros(self.dimx), np.zeros(self.dimx)
        y = np.zeros(self.nconstraints)
        mu = ctypes.c_double()
        _check(lib().v2g_get_state(self.h, _dp(x), _dp(y), _dp(z), ctypes.byref(mu)))
        return x, y, z, mu.value

    # -- maps -------------------------------------------------------------------
    def Au(self, u):
        u = np.ascontiguousarray(u, dtype=np.float64)
        assert u.size == self.dimx
        out = np.zeros(self.nconstraints)
        _check(lib().v2g_apply_A(self.h, _dp(u), _dp(out)))
        return out

    def ATu(self, u):
        u = np.ascontiguousarray(u, dtype=np.float64)
        assert u.size == self.nconstraints
        out = np.zeros(self.dimx)
        _check(lib().v2g_apply_AT(self.h, _dp(u), _dp(out)))
        return out

    def A_csr(self):
        """(rowptr, col, val) of A, built on the host."""
        L = lib()
        nnz = L.v2g_A_nnz(self.h)
        if nnz < 0:
            raise V2GError(V2G_ERR_UNSUPPORTED, "constraint table not available")
        rowptr = np.zeros(self.nconstraints + 1, dtype=np.int64)
        col = np.zeros(nnz, dtype=np.int32)
        val = np.zeros(nnz)
        _check(L.v2g_export_A(self.h, rowptr.ctypes.data_as(ctypes.POINTER(ctypes.c_long)), _ip(col), _dp(val)))
        return rowptr, col, val

    def map_batched_device(self, nvec, d_in, d_out, stream=None, transpose=False):
        """A (or A^T) on nvec instance-interleaved device vectors (raw pointers)."""
        f = lib().v2g_apply_AT_batched_device if transpose else lib().v2g_apply_A_batched_device
        _check(f(self.h, int(nvec), ctypes.c_void_p(d_in), ctypes.c_void_p(d_out),
                 ctypes.c_void_p(stream) if stream else None))

    def time_maps(self, nvec=1, reps=50):
        """(seconds per launch of A, of A^T) on nvec interleaved vectors (graph replay, CUDA events)."""
        a, t = ctypes.c_double(), ctypes.c_double()
        _check(lib().v2g_time_maps(self.h, int(nvec), int(reps), ctypes.byref(a), ctypes.byref(t)))
        return a.value, t.value

    def update_xz(self, mu):
        _check(lib().v2g_update_xz(self.h, float(mu)))

    def set_active_orbital_energies(self, energies):
        """Orbital energies of the active orbitals (Pitzer order); they number the
        spatial pairs as the plugin's orbital energies do."""
        e = np.ascontiguousarray(energies, dtype=np.float64)
        assert e.size == sum(self.active)
        _check(lib().v2g_set_active_orbital_energies(self.h, _dp(e)))

    def write_checkpoint(self, path):
        """Write mu, x, y, z (the plugin's checkpoint entries) to path."""
        _check(lib().v2g_write_checkpoint(self.h, os.fspath(path).encode()))

    def read_checkpoint(self, path):
        """Restore mu, x, y, z from a checkpoint of the same layout."""
        _check(lib().v2g_read_checkpoint(self.h, os.fspath(path).encode()))

    def pack_spatial_density(self, active_energies=None):
        """(d1, d2) handed to focas, as PackSpatialDensity (v2rdm_solver.cc:3664-3773)."""
        n1, n2 = ctypes.c_long(), ctypes.c_long()
        _check(lib().v2g_spatial_density_dims(self.h, ctypes.byref(n1), ctypes.byref(n2)))
        d1, d2 = np.zeros(n1.value), np.zeros(n2.value)
        e = None
        if active_energies is not None:
            e = np.ascontiguousarray(active_energies, dtype=np.float64)
            assert e.size == sum(self.active)
        _check(lib().v2g_pack_spatial_density(self.h, _dp(e) if e is not None else None, _dp(d1), _dp(d2)))
        return d1, d2

    def update_xz_noalloc(self, mu, d_c, d_y, d_x, d_z, stream=None):
        """Update_xz on caller-owned device vectors (raw pointers), allocating no
        device memory; for callers that cannot allocate (blocks <= 64 only)."""
        _check(lib().v2g_update_xz_noalloc(self.h, float(mu), ctypes.c_void_p(d_c), ctypes.c_void_p(d_y),
                                           ctypes.c_void_p(d_x), ctypes.c_void_p(d_z),
                                           ctypes.c_void_p(stream) if stream else None))

    # -- solve ------------------------------------------------------------------
    def compute_energy(self):
        """Runs the BPSDP loop; returns the total energy (raises if not converged)."""
        r = Result()
        code = lib().v2g_solve(self.h, ctypes.byref(r))
        self.result = r.as_dict()
        if code == V2G_ERR_NOT_CONVERGED:
            raise V2GError(code, "v2RDM did not converge.")
        _check(code)
        return r.e_total

    def solve_continue(self, max_outer):
        """Continues the BPSDP loop for at most max_outer outer iterations
        (v2g_solve_continue: one-step orbital optimisation segments); returns
        the result dict, with status V2G_ERR_NOT_CONVERGED when the segment
        ended unconverged."""
        r = Result()
        code = lib().v2g_solve_continue(self.h, int(max_outer), ctypes.byref(r))
        self.result = r.as_dict()
        if code not in (V2G_OK, V2G_ERR_NOT_CONVERGED):
            _check(code)
        return self.result

    def trace(self):
        L = lib()
        n = L.v2g_trace(self.h, None, 0)
        rows = np.zeros(8 * max(n, 1))
        L.v2g_trace(self.h, _dp(rows), n)
        return rows[: 8 * n].reshape(n, 8)


def block_gemm_device(dims, d_a, d_b, d_c, trans_a=False, trans_b=False, d_d=None, tensor_cores=True, device=0):
    """C_i = op(A_i) diag(d_i) op(B_i) for padded blocks on the device (pointers); see v2g_block_gemm_device."""
    dims = np.ascontiguousarray(dims, dtype=np.int32)
    _check(lib().v2g_block_gemm_device(len(dims), _ip(dims), ctypes.c_void_p(d_a), int(bool(trans_a)),
                                       ctypes.c_void_p(d_b), int(bool(trans_b)),
                                       ctypes.c_void_p(d_d) if d_d else None, ctypes.c_void_p(d_c),
                                       int(bool(tensor_cores)), int(device)))


def time_block_gemm(dims, d_a, d_b, d_c, tensor_cores=True, reps=20, device=0):
    """Seconds per product C_i = A_i B_i on the device (see v2g_time_block_gemm)."""
    dims = np.ascontiguousarray(dims, dtype=np.int32)
    sec = ctypes.c_double()
    _check(lib().v2g_time_block_gemm(len(dims), _ip(dims), ctypes.c_void_p(d_a), ctypes.c_void_p(d_b),
                                     ctypes.c_void_p(d_c), int(bool(tensor_cores)), int(reps), int(device),
                                     ctypes.byref(sec)))
    return sec.value


def _fp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


class WarmStart:
    """The learned warm start (v2g_ws_*): a pair-wise MLP trained on converged
    solutions of this solver that proposes D1, the D2ab pair diagonal and mu;
    a solver created with ``start="learned"`` projects the proposal onto
    A x = b at the start of its solve."""

    def __init__(self, hidden=224, device=0, seed=0):
        h = ctypes.c_void_p()
        _check(lib().v2g_ws_create(int(hidden), int(device), ctypes.c_ulonglong(seed), ctypes.byref(h)))
        self.h = h
        self.nparams = lib().v2g_ws_num_params(h)

    def __del__(self):
        h = getattr(self, "h", None)
        if h is not None and h.value and _lib is not None:
            _lib.v2g_ws_destroy(h)
            self.h = None

    @property
    def params(self):
        out = np.zeros(self.nparams, dtype=np.float32)
        _check(lib().v2g_ws_get_params(self.h, _fp(out)))
        return out

    @params.setter
    def params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        assert p.size == self.nparams
        _check(lib().v2g_ws_set_params(self.h, _fp(p)))

    @staticmethod
    def features(solver):
        rows = lib().v2g_ws_rows(solver.h)
        out = np.zeros((rows, 16), dtype=np.float32)
        _check(lib().v2g_ws_features(solver.h, _fp(out)))
        return out

    @staticmethod
    def targets(solver):
        rows = lib().v2g_ws_rows(solver.h)
        out = np.zeros((rows, 3), dtype=np.float32)
        _check(lib().v2g_ws_targets(solver.h, _fp(out)))
        return out

    def forward(self, features):
        f = np.ascontiguousarray(features, dtype=np.float32)
        out = np.zeros((f.shape[0], 3), dtype=np.float32)
        _check(lib().v2g_ws_forward(self.h, f.shape[0], _fp(f), _fp(out)))
        return out

    def gradient(self, features, targets):
        f = np.ascontiguousarray(features, dtype=np.float32)
        t = np.ascontiguousarray(targets, dtype=np.float32)
        g = np.zeros(self.nparams, dtype=np.float32)
        loss = ctypes.c_double()
        _check(lib().v2g_ws_gradient(self.h, f.shape[0], _fp(f), _fp(t), ctypes.byref(loss), _fp(g)))
        return loss.value, g

    def train(self, features, targets, epochs=100, batch_rows=4096, lr=1e-3):
        f = np.ascontiguousarray(features, dtype=np.float32)
        t = np.ascontiguousarray(targets, dtype=np.float32)
        loss = ctypes.c_double()
        _check(lib().v2g_ws_train(self.h, f.shape[0], _fp(f), _fp(t), int(epochs), int(batch_rows), float(lr),
                                  ctypes.byref(loss)))
        return loss.value

    def propose(self, solver, use_mu=True):
        """Writes the network's proposal into solver (a start="learned" solve);
        use_mu=False keeps mu = 1 with the proposed primal."""
        _check(lib().v2g_ws_propose(self.h, solver.h, int(bool(use_mu))))


def last_batch_stats():
    """Timing of the last solve on this thread (see v2g_batch_stats)."""
    st = BatchStats()
    _check(lib().v2g_last_batch_stats(ctypes.byref(st)))
    return st.as_dict()


def solve_batch(solvers):
    """Solves many problems in one GPU run; returns one result dict per solver."""
    n = len(solvers)
    hs = (ctypes.c_void_p * n)(*[s.h.value for s in solvers])
    res = (Result * n)()
    code = lib().v2g_solve_batch(hs, n, res)
    if code not in (V2G_OK, V2G_ERR_NOT_CONVERGED, V2G_ERR_NONFINITE):
        _check(code)
    out = [r.as_dict() for r in res]
    for s, r in zip(solvers, out):
        s.result = r
    return out
