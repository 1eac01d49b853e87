"""numpy restatement of the reference BPSDP hot path for C1 active spaces.

TEST INFRASTRUCTURE ONLY (the checker; the product never imports it).  It is
independent of both the compiled reference (oracle/_ref) and the product's
C++ row emitters: the constraint rows are re-derived here from the reference's
loops, assembled into a scipy sparse matrix, and the outer loop uses
numpy.linalg.eigh for Update_xz.  Pinned against the golden fixtures produced
by the compiled reference (tests/golden) in tests/test_cpu_oracle_port.py.

C1 index maps (basis.cc:439-548): geminal (p, q) has ab index q*n + p; the aa
geminals are the ab ones with p > q, numbered in the same order.
"""
import ctypes
import math

import numpy as np
import scipy.sparse as sp


class Layout:
    """Primal/dual layout of v2rdm_solver.cc:560-1270 for one irrep."""

    def __init__(self, n, na, nb, multiplicity=1, positivity="DQG", constrain_spin=True, constrain_sz=True):
        self.n, self.na, self.nb, self.mult = n, float(na), float(nb), multiplicity
        self.q2 = positivity in ("DQ", "DQG")
        self.g2 = positivity in ("DG", "DQG")
        if positivity not in ("D", "DQ", "DG", "DQG"):
            raise ValueError("the port covers D, DQ, DG and DQG")
        self.spin, self.sz = constrain_spin, constrain_sz
        self.singlet = na == nb
        self.aa_pairs = [(p, q) for q in range(n) for p in range(n) if p > q]  # basis.cc:531-545
        self.aa_index = {}
        for c, (p, q) in enumerate(self.aa_pairs):
            self.aa_index[(p, q)] = c
            self.aa_index[(q, p)] = c
        gab, gaa = n * n, len(self.aa_pairs)
        self.gab, self.gaa = gab, gaa
        blocks = [("d2ab", gab), ("d2aa", gaa), ("d2bb", gaa)]
        if self.spin:
            blocks.append(("d200", gab if self.singlet else 2 * gab))
        blocks += [("d1a", n), ("d1b", n), ("q1a", n), ("q1b", n)]
        if self.q2:
            blocks += [("q2ab", gab), ("q2aa", gaa), ("q2bb", gaa)]
        if self.g2:
            blocks += [("g2ab", gab), ("g2ba", gab), ("g2aa", 2 * gab)]
        self.blocks = blocks
        self.off = {}
        o = 0
        for name, d in blocks:
            self.off[name] = o
            o += d * d
        self.dimx = o
        self.dims = [d for _, d in blocks]

    def ab(self, p, q):
        return q * self.n + p

    def bas_ab(self, g):
        return g % self.n, g // self.n

    def aa(self, p, q):
        return self.aa_index[(p, q)]

    def el(self, fam, r, c, dim=None):
        d = dict(self.blocks)[fam] if dim is None else dim
        return self.off[fam] + r * d + c


def build_A(L):
    """Rows of A in the order of bpsdp_Au (v2rdm_solver.cc:3020-3065)."""
    rows, cols, vals = [], [], []
    nr = [0]

    def row(entries):
        for c, v in entries:
            rows.append(nr[0])
            cols.append(c)
            vals.append(v)
        nr[0] += 1

    n = L.n
    # D2_constraints_Au, d2.cc:296-547
    if L.sz:
        row([(L.el("d2ab", L.ab(i, j), L.ab(i, j)), 1.0) for i in range(n) for j in range(n)])
        for fam in ("d2aa", "d2bb"):
            row([(L.el(fam, L.aa(i, j), L.aa(i, j)), 1.0) for i in range(n) for j in range(n) if i != j])
    else:
        e = []
        for i in range(n):
            for j in range(n):
                e.append((L.el("d2ab", L.ab(i, j), L.ab(i, j)), 2.0))
                if i != j:
                    e.append((L.el("d2aa", L.aa(i, j), L.aa(i, j)), 1.0))
                    e.append((L.el("d2bb", L.aa(i, j), L.aa(i, j)), 1.0))
        row(e)
    for d1, q1 in (("d1a", "q1a"), ("d1b", "q1b")):
        for i in range(n):
            for j in range(n):
                row([(L.el(d1, j, i), 1.0), (L.el(q1, i, j), 1.0)])

    def sgn(a, k):
        return 1 if a < k else -1

    def contraction(d1, coef, spin_a, aa_fam):
        for i in range(n):
            for j in range(n):
                e = [(L.el(d1, i, j), coef)]
                if spin_a is not None:
                    for k in range(n):
                        ik = L.ab(i, k) if spin_a else L.ab(k, i)
                        jk = L.ab(j, k) if spin_a else L.ab(k, j)
                        e.append((L.el("d2ab", ik, jk), -1.0))
                if aa_fam is not None:
                    for k in range(n):
                        if k in (i, j):
                            continue
                        e.append((L.el(aa_fam, L.aa(i, k), L.aa(j, k)), -float(sgn(i, k) * sgn(j, k))))
                row(e)

    ntot = L.na + L.nb
    if not L.sz:
        contraction("d1a", ntot - 1.0, True, "d2aa")
        contraction("d1b", ntot - 1.0, False, "d2bb")
    else:
        contraction("d1a", L.nb, True, None)
        contraction("d1b", L.na, False, None)
        contraction("d1a", L.na - 1.0, None, "d2aa")
        contraction("d1b", L.nb - 1.0, None, "d2bb")
    # Spin_constraints_Au, spin.cc:274-493
    if L.spin:
        row([(L.el("d2ab", L.ab(i, j), L.ab(j, i)), 1.0) for i in range(n) for j in range(n)])
        r2 = math.sqrt(2.0)
        if L.singlet:
            for k in range(n * n):
                row([(L.off["d1a"] + k, 1.0), (L.off["d1b"] + k, -1.0)])
            for k in range(L.gaa * L.gaa):
                row([(L.off["d2aa"] + k, 1.0), (L.off["d2bb"] + k, -1.0)])
            for fam in ("d2aa", "d2bb"):
                for ij, (i, j) in enumerate(L.aa_pairs):
                    for kl, (k, l) in enumerate(L.aa_pairs):
                        row([(L.el(fam, ij, kl), 1.0),
                             (L.el("d2ab", L.ab(i, j), L.ab(k, l)), -0.5),
                             (L.el("d2ab", L.ab(j, i), L.ab(k, l)), 0.5),
                             (L.el("d2ab", L.ab(i, j), L.ab(l, k)), 0.5),
                             (L.el("d2ab", L.ab(j, i), L.ab(l, k)), -0.5)])
            for ij in range(L.gab):
                i, j = L.bas_ab(ij)
                for kl in range(L.gab):
                    k, l = L.bas_ab(kl)
                    w = -0.5 / ((r2 if i == j else 1.0) * (r2 if k == l else 1.0))
                    row([(L.el("d200", ij, kl), 1.0), (L.el("d2ab", ij, kl), w), (L.el("d2ab", L.ab(j, i), kl), w),
                         (L.el("d2ab", ij, L.ab(l, k)), w), (L.el("d2ab", L.ab(j, i), L.ab(l, k)), w)])
        else:
            g = L.gab
            for r in range(2 * g):
                for c in range(2 * g):
                    ij, kl = r % g, c % g
                    i, j = L.bas_ab(ij)
                    k, l = L.bas_ab(kl)
                    dij = r2 if i == j else 1.0
                    dkl = r2 if k == l else 1.0
                    if r < g and c < g:
                        a = b = cc = d = -0.5 / (dij * dkl)
                    elif r < g:
                        a, cc, b, d = -0.5 / dij, 0.5 / dij, -0.5 / dij, 0.5 / dij
                    elif c < g:
                        a, cc, b, d = -0.5 / dkl, -0.5 / dkl, 0.5 / dkl, 0.5 / dkl
                    else:
                        a, b, cc, d = -0.5, 0.5, 0.5, -0.5
                    row([(L.el("d200", r, c), 1.0), (L.el("d2ab", ij, kl), a), (L.el("d2ab", L.ab(j, i), kl), b),
                         (L.el("d2ab", ij, L.ab(l, k)), cc), (L.el("d2ab", L.ab(j, i), L.ab(l, k)), d)])
        if L.g2:
            for kl in range(L.gab):
                row([(L.el("g2ba", kl, L.ab(i, i)), 1.0) for i in range(n)])
            for kl in range(L.gab):
                row([(L.el("g2ba", L.ab(i, i), kl), 1.0) for i in range(n)])
    # Q2_constraints_Au, q2.cc:801-950
    if L.q2:
        for ij in range(L.gab):
            i, j = L.bas_ab(ij)
            for kl in range(L.gab):
                k, l = L.bas_ab(kl)
                e = [(L.el("d2ab", ij, kl), 1.0), (L.el("q2ab", ij, kl), -1.0)]
                if j == l:
                    e.append((L.el("d1a", k, i), -1.0))
                if i == k:
                    e.append((L.el("d1b", l, j), -1.0))
                row(e)
        for d2, q2, d1 in (("d2aa", "q2aa", "d1a"), ("d2bb", "q2bb", "d1b")):
            for ij, (i, j) in enumerate(L.aa_pairs):
                for kl, (k, l) in enumerate(L.aa_pairs):
                    e = [(L.el(d2, ij, kl), 1.0), (L.el(q2, ij, kl), -1.0)]
                    if j == l:
                        e.append((L.el(d1, k, i), -1.0))
                    if j == k:
                        e.append((L.el(d1, l, i), 1.0))
                    if i == l:
                        e.append((L.el(d1, k, j), 1.0))
                    if i == k:
                        e.append((L.el(d1, l, j), -1.0))
                    row(e)
    # G2_constraints_Au, g2.cc:1061-1260
    if L.g2:
        for g2, d1, swap in (("g2ab", "d1a", False), ("g2ba", "d1b", True)):
            for ij in range(L.gab):
                i, j = L.bas_ab(ij)
                for kl in range(L.gab):
                    k, l = L.bas_ab(kl)
                    e = [(L.el(g2, ij, kl), -1.0)]
                    if j == l:
                        e.append((L.el(d1, i, k), 1.0))
                    if not swap:
                        e.append((L.el("d2ab", L.ab(i, l), L.ab(k, j)), -1.0))
                    else:
                        e.append((L.el("d2ab", L.ab(l, i), L.ab(j, k)), -1.0))
                    row(e)
        g = L.gab
        for r in range(2 * g):
            for c in range(2 * g):
                ij, kl = r % g, c % g
                i, j = L.bas_ab(ij)
                k, l = L.bas_ab(kl)
                e = [(L.el("g2aa", r, c), -1.0)]
                if (r < g) == (c < g):
                    beta = r >= g
                    if j == l:
                        e.append((L.el("d1b" if beta else "d1a", i, k), 1.0))
                    if i != l and k != j:
                        s = sgn(i, l) * (1 if k < j else -1)
                        e.append((L.el("d2bb" if beta else "d2aa", L.aa(i, l), L.aa(k, j)), -float(s)))
                elif r < g:
                    e.append((L.el("d2ab", L.ab(i, l), L.ab(j, k)), 1.0))
                else:
                    e.append((L.el("d2ab", L.ab(l, i), L.ab(k, j)), 1.0))
                row(e)
    return sp.csr_matrix((vals, (rows, cols)), shape=(nr[0], L.dimx))


def build_b(L, ncon):
    """BuildConstraints, v2rdm_solver.cc:2518-3017."""
    b = np.zeros(ncon)
    n, o = L.n, 0
    if L.sz:
        b[0:3] = [L.na * L.nb, L.na * (L.na - 1.0), L.nb * (L.nb - 1.0)]
        o = 3
    else:
        t = L.na + L.nb
        b[0] = t * (t - 1.0)
        o = 1
    for _ in range(2):
        b[o:o + n * n] = np.eye(n).ravel()
        o += n * n
    o += (4 if L.sz else 2) * n * n
    if L.spin:
        ms = (L.mult - 1.0) / 2.0
        b[o] = 0.5 * (L.na + L.nb) + ms * ms - ms * (ms + 1.0)
        o += 1
        o += (n * n + 3 * L.gaa ** 2 + L.gab ** 2) if L.singlet else 4 * L.gab ** 2
        if L.g2:
            o += 2 * L.gab
    if L.q2:
        for ij in range(L.gab):
            i, j = L.bas_ab(ij)
            for kl in range(L.gab):
                k, l = L.bas_ab(kl)
                b[o + ij * L.gab + kl] = -float((i == k) and (j == l))
        o += L.gab ** 2
        for _ in range(2):
            for ij, (i, j) in enumerate(L.aa_pairs):
                for kl, (k, l) in enumerate(L.aa_pairs):
                    b[o + ij * L.gaa + kl] = -float((i == k) and (j == l)) + float((i == l) and (j == k))
            o += L.gaa ** 2
    return b


def build_c(L, h, eri):
    """RepackIntegrals / FrozenCoreEnergy for an all-active space (tei.cc:144-313):
    c[D2ab](ij,kl) = (ik|jl), c[D2aa/bb](ij,kl) = (ik|jl) - (il|jk), c[D1] = h."""
    c = np.zeros(L.dimx)
    n = L.n
    for ij in range(L.gab):
        i, j = L.bas_ab(ij)
        for kl in range(L.gab):
            k, l = L.bas_ab(kl)
            c[L.el("d2ab", ij, kl)] = eri[i, k, j, l]
    for ij, (i, j) in enumerate(L.aa_pairs):
        for kl, (k, l) in enumerate(L.aa_pairs):
            v = eri[i, k, j, l] - eri[i, l, j, k]
            c[L.el("d2aa", ij, kl)] = v
            c[L.el("d2bb", ij, kl)] = v
    c[L.off["d1a"]:L.off["d1a"] + n * n] = h.ravel()
    c[L.off["d1b"]:L.off["d1b"] + n * n] = h.ravel()
    return c


def random_guess(dimx, ncon):
    """Guess with TPDM_GUESS=RANDOM (v2rdm_solver.cc:2479-2490), glibc rand()."""
    libc = ctypes.CDLL("libc.so.6")
    libc.srand(0)
    rand = libc.rand
    rmax = 2147483647.0
    x = np.zeros(dimx)
    z = np.zeros(dimx)
    for i in range(dimx):
        x[i] = (rand() / rmax - 1.0) * 2.0
        z[i] = (rand() / rmax - 1.0) * 2.0
    y = np.array([(rand() / rmax - 1.0) * 2.0 for _ in range(ncon)])
    return x, y, z


def update_xz(A, L, x, y, c, mu):
    """Update_xz, v2rdm_solver.cc:3216-3289 (numpy eigh for Matrix::diagonalize)."""
    U = (A.T @ y - c) + mu * x
    xn = np.zeros_like(x)
    zn = np.zeros_like(x)
    o = 0
    for d in L.dims:
        M = U[o:o + d * d].reshape(d, d)
        M = 0.5 * (M + M.T)
        w, v = np.linalg.eigh(M)
        xn[o:o + d * d] = ((v * np.where(w > 0, w, 0.0) / mu) @ v.T).ravel()
        zn[o:o + d * d] = ((v * np.where(w < 0, -w, 0.0)) @ v.T).ravel()
        o += d * d
    return xn, zn


def cg(A, y, rhs, tol, maxiter, growth_stop=None):
    """CGSolver::solve, cg_solver.cc:125-177.

    growth_stop: the product's safeguard (None = the reference's CG): stop,
    keeping y, when p.Ap <= 0 or when r.r exceeds growth_stop times its
    smallest value in this solve (A A^T is singular, and a right-hand side
    with a null-space component above tol makes the plain iteration diverge).
    """
    r = rhs - A @ (A.T @ y)
    p = r.copy()
    it = 0
    rrmin = r @ r
    while True:
        Ap = A @ (A.T @ p)
        rr = r @ r
        pap = p @ Ap
        if growth_stop is not None and not pap > 0.0:
            break
        alpha = rr / pap
        y = y + alpha * p
        r = r - alpha * Ap
        rrnew = r @ r
        if math.sqrt(rrnew) < tol:
            break
        if growth_stop is not None:
            if rrnew > growth_stop * rrmin:
                break
            rrmin = min(rrmin, rrnew)
        p = (rrnew / rr) * p + r
        it += 1
        if it >= maxiter:
            break
    return y, it


def solve(L, A, b, c, x, y, z, r_conv, e_conv, maxiter=10000, cg_conv=1e-9, cg_maxiter=10000, tau=1.0,
          mu_update_frequency=500, cg_extrapolate=False, anderson_memory=0, cg_growth_stop=None):
    """The outer loop of v2rdm_solver.cc:1778-1908 (no orbital optimisation).

    cg_extrapolate: the product's option of that name; from the third outer
    iteration on, CG starts from y_k + (y_k - y_{k-1}) (the last two CG
    solutions) instead of y_k, with the same stopping test.

    anderson_memory: the product's option of that name (Anderson's method,
    type II, on w = (x, z)).  After each step g = (x', z') from w, f = g - w;
    with difference columns dF_j = f_{j+1} - f_j and dG_j = g_{j+1} - g_j of
    the last m steps, the next state is g - dG gamma, where
    (dF^T dF + 1e-10 tr(dF^T dF) I) gamma = dF^T f.  The stopping test and the
    energies are those of g; the history restarts from the current f whenever
    mu changes and when |f| more than doubled since the previous step (that
    step is then not mixed).
    """
    mu = 1.0
    ep = ed = 0.0
    oiter = 0
    iiter = 0
    starts = []  # the y each CG started from, before extrapolation
    hist_w, hist_f = [], []  # Anderson history: states and residuals
    fnorm_prev = None
    while True:
        x_in, z_in = x, z
        Ax = -tau * mu * (A @ x - b)
        z = c - z
        B = A @ z + Ax
        tol = 0.01 if oiter == 0 else 0.01 * min(ep, ed)
        tol = max(tol, cg_conv)
        if cg_extrapolate:
            y0 = y if len(starts) < 2 else y + (y - starts[-1])
            starts.append(y)
        else:
            y0 = y
        y, k = cg(A, y0, B, tol, cg_maxiter, growth_stop=cg_growth_stop)
        iiter += k
        w = np.concatenate([x_in, z_in]) if anderson_memory else None
        x, z = update_xz(A, L, x, y, c, mu)
        ed = np.linalg.norm(A.T @ y + z - c)
        ep = np.linalg.norm(A @ x - b)
        mu_changed = False
        if oiter % mu_update_frequency == 0 and oiter > 0:
            mu = mu * ep / ed
            mu_changed = True
        ep_energy, ed_energy = c @ x, b @ y
        oiter += 1
        if oiter == maxiter:
            return dict(converged=False, e_primal=ep_energy, e_dual=ed_energy, oiter=oiter, iiter=iiter, x=x, y=y,
                        z=z)
        if not (ep > r_conv or ed > r_conv or abs(ep_energy - ed_energy) > e_conv):
            return dict(converged=True, e_primal=ep_energy, e_dual=ed_energy, oiter=oiter, iiter=iiter, ep=ep, ed=ed,
                        x=x, y=y, z=z)
        if anderson_memory:
            g = np.concatenate([x, z])
            fnorm = np.linalg.norm(g - w)
            if mu_changed or (fnorm_prev is not None and fnorm > 2.0 * fnorm_prev):
                hist_w, hist_f = [], []
            fnorm_prev = fnorm
            hist_w.append(w)
            hist_f.append(g - w)
            if len(hist_w) > anderson_memory + 1:
                hist_w.pop(0)
                hist_f.pop(0)
            if len(hist_f) >= 2:
                dF = np.stack([hist_f[i + 1] - hist_f[i] for i in range(len(hist_f) - 1)], axis=1)
                dG = np.stack([(hist_w[i + 1] + hist_f[i + 1]) - (hist_w[i] + hist_f[i])
                               for i in range(len(hist_f) - 1)], axis=1)
                M = dF.T @ dF
                M = M + (1e-10 * np.trace(M) + 1e-300) * np.eye(M.shape[0])
                gamma = np.linalg.solve(M, dF.T @ hist_f[-1])
                g = g - dG @ gamma
                x, z = g[:L.dimx], g[L.dimx:]
