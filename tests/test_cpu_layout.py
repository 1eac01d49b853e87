"""CPU tests: the C ABI library loads and exports its header, and the host-side
layout, constraint table, b and c match the reference (golden fixtures made by
tests/golden/make_golden.py from the reference's own code, and the compiled
oracle when present)."""
import ctypes
import glob
import os
import re

import numpy as np
import pytest
import scipy.sparse as sp

from tests.helpers import GOLDEN, ROOT, csr_of, load, make_solver




def test_library_exports_every_header_symbol(v2g):
    header = open(os.path.join(ROOT, "include", "v2rdm_gpu.h")).read()
    declared = set(re.findall(r"\b(v2g_\w+)\s*\(", header))
    assert declared == set(v2g.EXPORTS)
    lib = v2g.lib()
    for name in declared:
        assert hasattr(lib, name), name


def test_sizes_match_reference_log(v2g):
    # tests/v2rdm8/output.ref:429-430: H2 (2,2), POSITIVITY D, C1 -> 50 variables, 51 constraints
    s = v2g.V2RDMSolver([2], 1, 1, options=dict(POSITIVITY="D"))
    assert (s.dimx, s.nconstraints) == (50, 51)
    # (10,10) DQG C1 and (20,20) DQG C1 sizes of the measured workloads
    s = v2g.V2RDMSolver([10], 5, 5)
    assert (s.dimx, s.nconstraints) == (98500, 91029)
    assert sorted(set(s.dimensions.tolist())) == [10, 45, 100, 200]


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "maps_*.npz"))),
                         ids=lambda p: os.path.basename(p))
def test_constraint_table_matches_golden(v2g, path):
    g = load(path)
    s = make_solver(v2g, g)
    assert s.dimx == int(g["dimx"]) and s.nconstraints == int(g["ncon"])
    assert s.dimensions.tolist() == g["block_dims"].tolist()
    A = csr_of(s)
    au, atw = A @ g["u"], A.T @ g["w"]
    assert np.abs(au - g["Au"]).max() <= 1e-13 * np.abs(g["Au"]).max()
    assert np.abs(atw - g["ATw"]).max() <= 1e-13 * np.abs(g["ATw"]).max()
    assert np.array_equal(s.b, g["b"])


def test_c_matches_golden(v2g):
    g = load(os.path.join(GOLDEN, "c_c2_core.npz"))
    docc, socc = g["docc"], g["socc"]
    na, nb = int(docc.sum() + socc.sum()), int(docc.sum())
    s = v2g.V2RDMSolver(g["amo"], na, nb, 1, frozen_docc=g["frzc"], restricted_docc=g["rstc"],
                        restricted_uocc=g["rstv"], frozen_uocc=g["frzv"])
    s.set_hamiltonian(g["oei"], g["qmo"], int(g["nq"]))
    assert np.abs(s.c - g["c"]).max() <= 1e-13 * np.abs(g["c"]).max()
    assert abs(s.efzc - float(g["efzc"])) <= 1e-12 * max(1.0, abs(float(g["efzc"])))


def test_oracle_reproduces_golden(ref):
    g = load(os.path.join(GOLDEN, "maps_c1_n4_dqg.npz"))
    r = ref.RefSolver(g["amopi"].tolist(), g["doccpi"].tolist(), soccpi=g["soccpi"].tolist(),
                      positivity=str(g["positivity"]))
    assert np.array_equal(r.Au(g["u"]), g["Au"])
    assert np.array_equal(r.ATu(g["w"]), g["ATw"])


@pytest.mark.parametrize("spec", [
    ([7], 3, 3, 1, "DQG"), ([6], 3, 2, 2, "DQG"), ([3, 3], 3, 3, 1, "DQG"), ([2, 2, 2, 1], 3, 3, 1, "DQ"),
    ([4], 2, 2, 1, "DQGT1"), ([5], 3, 2, 2, "DQGT1T2"), ([3, 2], 3, 2, 2, "DQGT2"), ([2, 2, 1, 1], 3, 3, 1, "DQGT"),
])
def test_constraint_table_matches_oracle(v2g, ref, spec):
    amopi, na, nb, mult, pos = spec
    docc = [0] * len(amopi)
    socc = [0] * len(amopi)
    # distribute electrons over irreps (only the totals matter for the layout)
    left_b, left_s = nb, na - nb
    for h in range(len(amopi)):
        d = min(amopi[h], left_b)
        docc[h] = d
        left_b -= d
        s_ = min(amopi[h] - d, left_s)
        socc[h] = s_
        left_s -= s_
    r = ref.RefSolver(amopi, docc, soccpi=socc, multiplicity=mult, positivity=pos)
    s = v2g.V2RDMSolver(amopi, na, nb, mult, options=dict(POSITIVITY=pos))
    A = csr_of(s)
    rng = np.random.default_rng(5)
    u, w = rng.standard_normal(s.dimx), rng.standard_normal(s.nconstraints)
    a = r.Au(u)
    t = r.ATu(w)
    assert np.abs(A @ u - a).max() <= 1e-13 * np.abs(a).max()
    assert np.abs(A.T @ w - t).max() <= 1e-13 * np.abs(t).max()


@pytest.mark.parametrize("spec", [
    ([4], 2, "DQG", True, False, True), ([5], 2, "DQG", True, True, False), ([3, 2], 2, "DQG", True, False, True),
    ([2, 2, 1, 1], 3, "DQG", True, True, False), ([5], 2, "DG", False, True, False),
])
def test_spin_adapted_tables_match_oracle(v2g, ref, spec):
    # SPIN_ADAPT_Q2 / SPIN_ADAPT_G2 (q2.cc:260-468, g2.cc:235-455); the oracle's
    # orbital energies are given in Pitzer order, the order the layout assumes
    amopi, nb, pos, saq2, sag2, spin = spec
    docc, left = [], nb
    for a in amopi:
        docc.append(min(a, left))
        left -= docc[-1]
    r = ref.RefSolver(amopi, docc, positivity=pos, constrain_spin=spin, energies=np.arange(sum(amopi), dtype=float),
                      spin_adapt_q2=saq2, spin_adapt_g2=sag2)
    s = v2g.V2RDMSolver(amopi, nb, nb, 1, options=dict(POSITIVITY=pos, CONSTRAIN_SPIN=spin, SPIN_ADAPT_Q2=saq2,
                                                        SPIN_ADAPT_G2=sag2))
    assert (s.dimx, s.nconstraints) == (r.dimx, r.ncon)
    assert list(s.dimensions) == list(r.block_dims)
    A = csr_of(s)
    rng = np.random.default_rng(7)
    u, w = rng.standard_normal(s.dimx), rng.standard_normal(s.nconstraints)
    a, t = r.Au(u), r.ATu(w)
    assert np.abs(A @ u - a).max() <= 1e-13 * np.abs(a).max()
    assert np.abs(A.T @ w - t).max() <= 1e-13 * np.abs(t).max()
    r.build_constraints()
    assert np.array_equal(s.b, r.get("b"))


@pytest.mark.parametrize("spec", [
    ([4], 2, 2, 1, "DQG", True), ([5], 3, 2, 2, "DQG", True), ([6], 3, 3, 1, "D", False),
    ([2, 2, 1, 1], 3, 3, 1, "DQG", True), ([4], 1, 1, 1, "DQG", True), ([5], 3, 1, 3, "DQG", True),
])
def test_d3_tables_match_oracle(v2g, ref, spec):
    # CONSTRAIN_D3 (d3.cc:57-298): families depend on the active electron counts
    amopi, na, nb, mult, pos, spin = spec
    docc, socc, lb, ls = [], [], nb, na - nb
    for a in amopi:
        docc.append(min(a, lb))
        lb -= docc[-1]
        socc.append(min(a - docc[-1], ls))
        ls -= socc[-1]
    r = ref.RefSolver(amopi, docc, soccpi=socc, multiplicity=mult, positivity=pos, constrain_spin=spin,
                      constrain_d3=True)
    s = v2g.V2RDMSolver(amopi, na, nb, mult, options=dict(POSITIVITY=pos, CONSTRAIN_SPIN=spin, CONSTRAIN_D3=True))
    assert (s.dimx, s.nconstraints) == (r.dimx, r.ncon)
    assert list(s.dimensions) == list(r.block_dims)
    A = csr_of(s)
    rng = np.random.default_rng(11)
    u, w = rng.standard_normal(s.dimx), rng.standard_normal(s.nconstraints)
    a, t = r.Au(u), r.ATu(w)
    assert np.abs(A @ u - a).max() <= 1e-13 * np.abs(a).max()
    assert np.abs(A.T @ w - t).max() <= 1e-13 * np.abs(t).max()
    r.build_constraints()
    assert np.array_equal(s.b, r.get("b"))


@pytest.mark.parametrize("spec", [
    ([4], 2, 2, 1, "DQG", True), ([5], 3, 2, 2, "DQG", True), ([6], 4, 4, 1, "D", False),
    ([2, 2, 1, 1], 3, 3, 1, "DQG", True), ([5], 4, 1, 4, "D", True),
])
def test_d4_tables_match_oracle(v2g, ref, spec):
    # CONSTRAIN_D4 (d4.cc:55-312, quartets basis.cc:758-904), including the two
    # empty blocks the reference's constraint count adds at the end
    amopi, na, nb, mult, pos, spin = spec
    docc, socc, lb, ls = [], [], nb, na - nb
    for a in amopi:
        docc.append(min(a, lb))
        lb -= docc[-1]
        socc.append(min(a - docc[-1], ls))
        ls -= socc[-1]
    r = ref.RefSolver(amopi, docc, soccpi=socc, multiplicity=mult, positivity=pos, constrain_spin=spin,
                      constrain_d4=True)
    s = v2g.V2RDMSolver(amopi, na, nb, mult, options=dict(POSITIVITY=pos, CONSTRAIN_SPIN=spin, CONSTRAIN_D4=True))
    assert (s.dimx, s.nconstraints) == (r.dimx, r.ncon)
    assert list(s.dimensions) == list(r.block_dims)
    A = csr_of(s)
    rng = np.random.default_rng(13)
    u, w = rng.standard_normal(s.dimx), rng.standard_normal(s.nconstraints)
    a, t = r.Au(u), r.ATu(w)
    assert np.abs(A @ u - a).max() <= 1e-13 * np.abs(a).max()
    assert np.abs(A.T @ w - t).max() <= 1e-13 * np.abs(t).max()
    r.build_constraints()
    assert np.array_equal(s.b, r.get("b"))


def test_spin_adaptation_restrictions(v2g):
    # v2rdm_solver.cc:538-558: not with T1/T2, not for S = M != 0
    with pytest.raises(v2g.V2GError):
        v2g.V2RDMSolver([4], 2, 2, options=dict(POSITIVITY="DQGT2", SPIN_ADAPT_Q2=True))
    with pytest.raises(v2g.V2GError):
        v2g.V2RDMSolver([4], 3, 1, 3, options=dict(SPIN_ADAPT_G2=True, CONSTRAIN_SPIN=False))


def test_invalid_options_fail_loudly(v2g):
    with pytest.raises(v2g.V2GError):
        v2g.V2RDMSolver([4], 2, 2, options=dict(POSITIVITY="DQX"))
    with pytest.raises(v2g.V2GError):
        v2g.V2RDMSolver([4], 2, 2, options=dict(MAXITER=0))
    with pytest.raises(KeyError):
        v2g.V2RDMSolver([4], 2, 2, options=dict(NOT_AN_OPTION=1))


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "pack_*.npz"))),
                         ids=lambda p: os.path.basename(p))
def test_oracle_reproduces_spatial_density_golden(ref, path):
    g = load(path)
    e = g["energies"] if g["energies"].size else None
    r = ref.RefSolver(g["amopi"].tolist(), g["doccpi"].tolist(), soccpi=g["soccpi"].tolist(),
                      multiplicity=int(g["soccpi"].sum()) + 1, energies=e)
    r.set("x", g["x"])
    d1, d2 = r.pack_spatial_density()
    assert np.array_equal(d1, g["d1"]) and np.array_equal(d2, g["d2"])


def test_spatial_density_dims(v2g):
    for amopi, na, nb in (([4], 2, 2), ([2, 1, 1, 2], 2, 2), ([3, 2], 3, 2)):
        s = v2g.V2RDMSolver(amopi, na, nb, na - nb + 1)
        n1, n2 = ctypes.c_long(), ctypes.c_long()
        assert v2g.lib().v2g_spatial_density_dims(s.h, ctypes.byref(n1), ctypes.byref(n2)) == 0
        n = sum(amopi)
        assert n1.value == sum(a * (a + 1) // 2 for a in amopi)
        # spatial pairs i >= j per irrep of the pair
        sym = [h for h, a in enumerate(amopi) for _ in range(a)]
        g00 = [0] * len(amopi)
        for i in range(n):
            for j in range(i + 1):
                g00[sym[i] ^ sym[j]] += 1
        assert n2.value == sum(g * (g + 1) // 2 for g in g00)


@pytest.mark.parametrize("amopi,energies", [
    ([2, 1, 1, 2], [0.3, 1.1, 0.2, 0.5, 0.1, 0.9]), ([3, 2], [0.2, 0.4, 0.9, 0.3, 0.35]),
    ([5], [0.5, 0.1, 0.3, 0.3, 0.2]),
])
def test_spin_adapted_q2_follows_orbital_energies(v2g, ref, amopi, energies):
    # the singlet Q2 block is numbered by spatial pairs in orbital-energy order
    nb = sum(amopi) // 2
    docc, left = [], nb
    for a in amopi:
        docc.append(min(a, left))
        left -= docc[-1]
    r = ref.RefSolver(amopi, docc, energies=energies, spin_adapt_q2=True)
    s = v2g.V2RDMSolver(amopi, nb, nb, options=dict(SPIN_ADAPT_Q2=True))
    s.set_active_orbital_energies(energies)
    A = csr_of(s)
    rng = np.random.default_rng(17)
    u = rng.standard_normal(s.dimx)
    a = r.Au(u)
    assert np.abs(A @ u - a).max() <= 1e-13 * np.abs(a).max()
