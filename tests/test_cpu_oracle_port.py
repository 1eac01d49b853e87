"""The numpy restatement in oracle/port.py against the reference's own outputs
(golden fixtures from the compiled reference) and against the product's
constraint table (CPU only)."""
import os

import numpy as np
import pytest

from oracle import port
from tests.helpers import GOLDEN, csr_of, load


@pytest.mark.parametrize("name", ["c1_n4_dqg", "c1_n6_dqg", "c1_n5_triplet_dqg", "c1_n5_dqg_nosz", "c1_n4_d"])
def test_port_maps_match_reference(name):
    g = load(os.path.join(GOLDEN, f"maps_{name}.npz"))
    docc, socc = g["doccpi"], g["soccpi"]
    na, nb = int(docc.sum() + socc.sum()), int(docc.sum())
    L = port.Layout(int(g["amopi"][0]), na, nb, int(socc.sum()) + 1, str(g["positivity"]),
                    bool(g["constrain_spin"]), bool(g["constrain_sz"]))
    A = port.build_A(L)
    assert A.shape == (int(g["ncon"]), int(g["dimx"]))
    assert L.dims == g["block_dims"].tolist()
    assert np.abs(A @ g["u"] - g["Au"]).max() <= 1e-13 * np.abs(g["Au"]).max()
    assert np.abs(A.T @ g["w"] - g["ATw"]).max() <= 1e-13 * np.abs(g["ATw"]).max()
    assert np.array_equal(port.build_b(L, A.shape[0]), g["b"])


def test_port_guess_matches_reference_start():
    g = load(os.path.join(GOLDEN, "solve_synthetic_n4_s0.npz"))
    L = port.Layout(4, 2, 2)
    A = port.build_A(L)
    x, y, z = port.random_guess(L.dimx, A.shape[0])
    # the reference's first iteration line starts from this state: check its
    # primal energy against the trace is not possible without c; check the
    # guess range and determinism instead
    x2, y2, z2 = port.random_guess(L.dimx, A.shape[0])
    assert np.array_equal(x, x2) and x.min() >= -2.0 and x.max() <= 0.0


def test_port_solve_matches_reference():
    from v2rdm_casscf_b200.hamiltonian import synthetic

    g = load(os.path.join(GOLDEN, "solve_synthetic_n4_s0.npz"))
    a = synthetic(4, int(g["seed"]))
    L = port.Layout(4, a.na, a.nb)
    A = port.build_A(L)
    b = port.build_b(L, A.shape[0])
    c = port.build_c(L, a.h, a.eri())
    x, y, z = port.random_guess(L.dimx, A.shape[0])
    out = port.solve(L, A, b, c, x, y, z, float(g["r_conv"]), float(g["e_conv"]))
    assert out["converged"]
    assert abs(out["e_primal"] - float(g["e_primal"])) <= 1e-6


def test_port_cg_extrapolation_same_energy_fewer_cg_iterations():
    # the product's cg_extrapolate option, restated in the port: the stopping
    # test is unchanged, so the converged energy is the reference's while CG
    # needs far fewer iterations (about half at n = 4..8)
    from v2rdm_casscf_b200.hamiltonian import synthetic

    g = load(os.path.join(GOLDEN, "solve_synthetic_n4_s0.npz"))
    a = synthetic(4, int(g["seed"]))
    L = port.Layout(4, a.na, a.nb)
    A = port.build_A(L)
    b = port.build_b(L, A.shape[0])
    c = port.build_c(L, a.h, a.eri())
    runs = []
    for ex in (False, True):
        x, y, z = port.random_guess(L.dimx, A.shape[0])
        runs.append(port.solve(L, A, b, c, x, y, z, float(g["r_conv"]), float(g["e_conv"]), cg_extrapolate=ex))
    plain, extr = runs
    assert plain["converged"] and extr["converged"]
    assert abs(extr["e_primal"] - float(g["e_primal"])) <= 1e-6
    assert abs(extr["oiter"] - plain["oiter"]) <= 0.05 * plain["oiter"]
    assert extr["iiter"] <= 0.7 * plain["iiter"]


@pytest.mark.parametrize("m", [5, 10])
def test_port_anderson_same_energy_fewer_outer_iterations(m):
    # the product's anderson_memory option, restated in the port: same
    # stopping test on the plain step, so the reference's energy, in a
    # fraction of the outer iterations (about 2-5x fewer at n = 4..8)
    from v2rdm_casscf_b200.hamiltonian import synthetic

    g = load(os.path.join(GOLDEN, "solve_synthetic_n4_s0.npz"))
    a = synthetic(4, int(g["seed"]))
    L = port.Layout(4, a.na, a.nb)
    A = port.build_A(L)
    b = port.build_b(L, A.shape[0])
    c = port.build_c(L, a.h, a.eri())
    x, y, z = port.random_guess(L.dimx, A.shape[0])
    out = port.solve(L, A, b, c, x, y, z, float(g["r_conv"]), float(g["e_conv"]), anderson_memory=m)
    assert out["converged"]
    assert abs(out["e_primal"] - float(g["e_primal"])) <= 1e-6
    assert out["oiter"] <= 0.6 * int(g["oiter"])


def test_port_anderson_guard_on_a_stretched_chain():
    # H4 at 1.5 A: without the residual-growth restart, Anderson mixing needs
    # more outer iterations than no mixing; with it (the product's rule), far
    # fewer, at the same energy
    from v2rdm_casscf_b200.hchain import hydrogen_chain

    a = hydrogen_chain(4, 1.5)
    L = port.Layout(a.n, a.na, a.nb)
    A = port.build_A(L).tocsr()
    b = port.build_b(L, A.shape[0])
    c = port.build_c(L, a.h, a.eri())
    w, _ = port.cg(A, np.zeros(A.shape[0]), b, 1e-10 * np.linalg.norm(b), 20000)
    x0 = A.T @ w
    runs = [port.solve(L, A, b, c, x0.copy(), np.zeros(A.shape[0]), np.zeros(L.dimx), 1e-6, 1e-7, cg_extrapolate=True,
                       anderson_memory=m) for m in (0, 10)]
    assert all(r["converged"] for r in runs)
    assert abs(runs[1]["e_primal"] - runs[0]["e_primal"]) <= 1e-6
    assert runs[1]["oiter"] <= 0.5 * runs[0]["oiter"]


def test_port_agrees_with_product_table(v2g):
    L = port.Layout(5, 3, 2, 2)
    A = port.build_A(L)
    s = v2g.V2RDMSolver([5], 3, 2, 2)
    P = csr_of(s)
    assert (A - P).count_nonzero() == 0 or abs(A - P).max() <= 1e-15


def test_port_accelerated_configuration_on_a_chain():
    # the bench's --accelerated loop options (Anderson memory 10, extrapolated
    # CG start, MU_UPDATE_FREQUENCY 250) on H4 at 1.0 A: the plain loop's
    # energy in a fraction of its outer and CG iterations
    from v2rdm_casscf_b200.hchain import hydrogen_chain

    a = hydrogen_chain(4, 1.0)
    L = port.Layout(a.n, a.na, a.nb)
    A = port.build_A(L).tocsr()
    b = port.build_b(L, A.shape[0])
    c = port.build_c(L, a.h, a.eri())
    w, _ = port.cg(A, np.zeros(A.shape[0]), b, 1e-10 * np.linalg.norm(b), 20000)
    runs = [port.solve(L, A, b, c, A.T @ w, np.zeros(A.shape[0]), np.zeros(L.dimx), 1e-6, 1e-7, **kw)
            for kw in ({}, dict(anderson_memory=10, cg_extrapolate=True, mu_update_frequency=250))]
    assert all(r["converged"] for r in runs)
    assert abs(runs[1]["e_primal"] - runs[0]["e_primal"]) <= 1e-6
    assert runs[1]["oiter"] <= 0.6 * runs[0]["oiter"]
    assert runs[1]["iiter"] <= 0.6 * runs[0]["iiter"]
