"""GPU parity tests through the C ABI against the reference.

Golden fixtures come from the reference's own code (tests/golden/make_golden.py);
when the compiled oracle is present it is also run on fresh seeds.
Tolerances: the maps are FP64 gathers, within 1e-12 relative;
the projection within 1e-10 relative to the block norms (eigensolvers differ);
total energies within 1e-6 Eh of the reference at the same convergence
thresholds.
"""
import glob
import os

import numpy as np
import pytest

from tests.helpers import GOLDEN, load, make_solver

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "maps_*.npz"))),
                         ids=lambda p: os.path.basename(p))
def test_maps_match_reference(v2g, path):
    g = load(path)
    s = make_solver(v2g, g)
    au = s.Au(g["u"])
    atw = s.ATu(g["w"])
    assert np.abs(au - g["Au"]).max() <= 1e-12 * np.abs(g["Au"]).max()
    assert np.abs(atw - g["ATw"]).max() <= 1e-12 * np.abs(g["ATw"]).max()


def test_maps_adjoint(v2g):
    s = v2g.V2RDMSolver([8], 4, 4)
    rng = np.random.default_rng(0)
    u, w = rng.standard_normal(s.dimx), rng.standard_normal(s.nconstraints)
    lhs = np.dot(s.Au(u), w)
    rhs = np.dot(u, s.ATu(w))
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs)


@pytest.mark.parametrize("n", [4, 6])
def test_update_xz_matches_reference(v2g, n):
    # n=4: every block <= 64 (shared-memory Jacobi); n=6: G2 block of 72 (block Jacobi)
    from v2rdm_casscf_b200.hamiltonian import synthetic

    g = load(os.path.join(GOLDEN, f"xz_n{n}.npz"))
    a = synthetic(n, int(g["seed"]))
    s = v2g.V2RDMSolver.from_active_space(a)
    s.set_state(g["x"], g["y"], g["z"], float(g["mu"]))
    s.update_xz(float(g["mu"]))
    x, y, z, _ = s.get_state()
    scale = max(np.abs(g["x_out"]).max(), np.abs(g["z_out"]).max())
    assert np.abs(x - g["x_out"]).max() <= 1e-10 * scale
    assert np.abs(z - g["z_out"]).max() <= 1e-10 * scale


def _solve_golden(v2g, name):
    from v2rdm_casscf_b200.hamiltonian import synthetic

    g = load(os.path.join(GOLDEN, f"solve_{name}.npz"))
    a = synthetic(int(g["n"]), int(g["seed"]), electrons=int(g["electrons"]))
    pos = str(g["positivity"]) if "positivity" in g else "DQG"
    saq2 = bool(g["spin_adapt_q2"]) if "spin_adapt_q2" in g else False
    s = v2g.V2RDMSolver.from_active_space(
        a, options=dict(R_CONVERGENCE=float(g["r_conv"]), E_CONVERGENCE=float(g["e_conv"]), POSITIVITY=pos,
                        SPIN_ADAPT_Q2=saq2),
        record_trace=True)
    s.guess()
    return g, s


@pytest.mark.parametrize("name", ["synthetic_n4_s0", "synthetic_n4_s1", "synthetic_n5_s2", "synthetic_n5_s2_doublet",
                                  "synthetic_n4_s1_dqgt1", "synthetic_n4_s0_saq2"])
def test_solve_matches_reference(v2g, name):
    # Converged energies agree; individual iterations do not have to, since CG
    # on A A^T from the random start amplifies rounding (a sparse vs dense
    # matvec on the CPU already moves iteration 0 by 5e-5 Eh).
    g, s = _solve_golden(v2g, name)
    e = s.compute_energy()
    r = s.result
    assert r["status"] == 0
    assert abs(e - float(g["e_primal"])) <= 1e-6
    assert abs(r["e_dual"] - float(g["e_dual"])) <= 1e-6
    assert r["ep"] <= float(g["r_conv"]) and r["ed"] <= float(g["r_conv"])
    assert abs(r["oiter"] - int(g["oiter"])) <= 0.25 * int(g["oiter"])
    tr = s.trace()
    assert len(tr) == r["oiter"]
    assert np.all(np.diff(tr[:, 0]) == 1)


def test_batch_equals_individual_solves(v2g):
    g0, s0 = _solve_golden(v2g, "synthetic_n4_s0")
    g1, s1 = _solve_golden(v2g, "synthetic_n4_s1")
    g2, s2 = _solve_golden(v2g, "synthetic_n5_s2")  # another layout in the same call
    # looser thresholds for one instance: options are per instance
    from v2rdm_casscf_b200.hamiltonian import synthetic

    s3 = v2g.V2RDMSolver.from_active_space(synthetic(4, 1), options=dict(R_CONVERGENCE=1e-4, E_CONVERGENCE=1e-4))
    s3.guess()
    res = v2g.solve_batch([s0, s1, s2, s3])
    assert all(r["status"] == 0 for r in res)
    for r, g in zip(res[:3], (g0, g1, g2)):
        assert abs(r["e_total"] - float(g["e_primal"])) <= 1e-6
    assert res[3]["oiter"] < res[1]["oiter"]
    g1b, s1b = _solve_golden(v2g, "synthetic_n4_s1")
    e1 = s1b.compute_energy()
    # the per-instance reductions sum in an order that depends on the group
    # size, so batch and single solves agree to rounding, not bit for bit
    assert abs(e1 - res[1]["e_total"]) <= 1e-9
    assert abs(s1b.result["oiter"] - res[1]["oiter"]) <= 0.02 * res[1]["oiter"]


def test_solve_matches_oracle_fresh_seed(v2g, ref):
    from v2rdm_casscf_b200.hamiltonian import synthetic

    a2 = synthetic(5, 11, electrons=5)  # doublet (5e,5o)
    opts = dict(R_CONVERGENCE=1e-6, E_CONVERGENCE=1e-7)
    r = ref.RefSolver([5], [2], soccpi=[1], multiplicity=2, positivity="DQG", r_convergence=1e-6,
                      e_convergence=1e-7)
    r.set_integrals(a2.oei_packed, a2.qmo, a2.nq)
    r.guess()
    r.build_constraints()
    out = r.solve()
    s = v2g.V2RDMSolver.from_active_space(a2, options=opts)
    s.guess()
    e = s.compute_energy()
    assert out["converged"]
    assert abs(e - out["e_primal"]) <= 1e-6


@pytest.mark.parametrize("name", ["synthetic_n4_s1", "synthetic_n5_s2", "synthetic_n5_s2_doublet"])
def test_adaptive_projection_reaches_the_same_energy(v2g, name):
    # loose eigendecompositions far from the solution, exact ones near it:
    # same converged energy as the reference within the parity tolerance
    from v2rdm_casscf_b200.hamiltonian import synthetic

    g = load(os.path.join(GOLDEN, f"solve_{name}.npz"))
    a = synthetic(int(g["n"]), int(g["seed"]), electrons=int(g["electrons"]))
    s = v2g.V2RDMSolver.from_active_space(
        a, options=dict(R_CONVERGENCE=float(g["r_conv"]), E_CONVERGENCE=float(g["e_conv"])), projection="adaptive")
    s.guess()
    e = s.compute_energy()
    assert s.result["status"] == 0
    assert abs(e - float(g["e_primal"])) <= 1e-6
    assert s.result["ep"] <= float(g["r_conv"]) and s.result["ed"] <= float(g["r_conv"])


def test_adaptive_projection_with_large_blocks(v2g):
    # (6e,6o): 72 x 72 G2 block takes the refinement / block-Jacobi path
    from v2rdm_casscf_b200.hamiltonian import synthetic

    a = synthetic(6, 4)
    opts = dict(R_CONVERGENCE=1e-6, E_CONVERGENCE=1e-7)
    s1 = v2g.V2RDMSolver.from_active_space(a, options=opts)
    s1.guess()
    e1 = s1.compute_energy()
    s2 = v2g.V2RDMSolver.from_active_space(a, options=opts, projection="adaptive")
    s2.guess()
    e2 = s2.compute_energy()
    assert s1.result["status"] == 0 and s2.result["status"] == 0
    assert abs(e1 - e2) <= 1e-6


def test_cg_tolerance_factor_reaches_the_same_energy(v2g):
    from v2rdm_casscf_b200.hamiltonian import synthetic

    g = load(os.path.join(GOLDEN, "solve_synthetic_n5_s2.npz"))
    a = synthetic(int(g["n"]), int(g["seed"]), electrons=int(g["electrons"]))
    s = v2g.V2RDMSolver.from_active_space(
        a, options=dict(R_CONVERGENCE=float(g["r_conv"]), E_CONVERGENCE=float(g["e_conv"])), projection="adaptive",
        cg_tolerance_factor=0.1)
    s.guess()
    e = s.compute_energy()
    assert s.result["status"] == 0
    assert abs(e - float(g["e_primal"])) <= 1e-6
    assert s.result["iiter"] < int(g["iiter"])


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "pack_*.npz"))),
                         ids=lambda p: os.path.basename(p))
def test_spatial_density_matches_reference(v2g, path):
    # PackSpatialDensity: the same sums in the same order, so bit for bit
    g = load(path)
    amopi = g["amopi"].tolist()
    na = int(g["doccpi"].sum() + g["soccpi"].sum())
    nb = int(g["doccpi"].sum())
    s = v2g.V2RDMSolver(amopi, na, nb, na - nb + 1)
    s.set_state(g["x"], np.zeros(s.nconstraints), np.zeros(s.dimx), 1.0)
    e = g["energies"] if g["energies"].size else None
    d1, d2 = s.pack_spatial_density(e)
    assert np.array_equal(d1, g["d1"])
    assert np.array_equal(d2, g["d2"])


@pytest.mark.parametrize("n,seed", [(3, 0), (4, 1), (5, 2)])
def test_two_electron_d_equals_fci(v2g, n, seed):
    # known answer independent of the reference: D is exact for two electrons
    from tests.helpers import fci_two_electron_singlet
    from v2rdm_casscf_b200.hamiltonian import synthetic

    a = synthetic(n, seed, electrons=2)
    s = v2g.V2RDMSolver.from_active_space(a, options=dict(POSITIVITY="D", R_CONVERGENCE=1e-7, E_CONVERGENCE=1e-8))
    s.guess()
    e = s.compute_energy()
    assert abs(e - fci_two_electron_singlet(a)) <= 1e-6


def test_h10_chain_matches_reference(v2g):
    # the CPU-runnable workload: linear H10, 0.9 A, STO-3G RHF orbitals, all
    # active, DQG; integrals stored with the reference's converged energy
    from v2rdm_casscf_b200.hamiltonian import ActiveSpace

    g = load(os.path.join(GOLDEN, "solve_h10_chain.npz"))
    a = ActiveSpace(g["h"], g["L"], 5, 5, enuc=float(g["enuc"]))
    s = v2g.V2RDMSolver.from_active_space(
        a, options=dict(R_CONVERGENCE=float(g["r_conv"]), E_CONVERGENCE=float(g["e_conv"])))
    s.guess()
    e = s.compute_energy()
    assert abs(e - float(g["e_primal"])) <= 1e-6
    assert e < float(g["scf_energy"])  # a lower bound below the RHF energy
    assert abs(s.result["oiter"] - int(g["oiter"])) <= 0.25 * int(g["oiter"])


@pytest.mark.parametrize("n,seed", [(4, 0), (4, 1), (5, 2)])
def test_three_electron_d_d3_equals_fci(v2g, n, seed):
    # known answer independent of the reference: D + D3 is exact for three electrons
    from tests.helpers import fci_spin_state
    from v2rdm_casscf_b200.hamiltonian import synthetic

    a = synthetic(n, seed, electrons=3)
    s = v2g.V2RDMSolver.from_active_space(
        a, options=dict(POSITIVITY="D", CONSTRAIN_D3=True, R_CONVERGENCE=1e-7, E_CONVERGENCE=1e-8))
    s.guess()
    e = s.compute_energy()
    assert abs(e - fci_spin_state(a, 2)) <= 1e-6


@pytest.mark.parametrize("seed", [0, 1])
def test_four_electron_d_d4_equals_fci(v2g, seed):
    # known answer independent of the reference: D + D3 + D4 is exact for four electrons
    from tests.helpers import fci_spin_state
    from v2rdm_casscf_b200.hamiltonian import synthetic

    a = synthetic(4, seed, electrons=4)
    s = v2g.V2RDMSolver.from_active_space(
        a, options=dict(POSITIVITY="D", CONSTRAIN_D4=True, R_CONVERGENCE=1e-7, E_CONVERGENCE=1e-8))
    s.guess()
    e = s.compute_energy()
    assert abs(e - fci_spin_state(a, 1)) <= 1e-6


@pytest.mark.parametrize("name", ["synthetic_n4_s0", "synthetic_n5_s2_doublet"])
def test_feasible_start_reaches_reference_energy(v2g, name):
    # the least-norm feasible start (start="feasible") changes the path, not the answer
    from v2rdm_casscf_b200.hamiltonian import synthetic

    g = load(os.path.join(GOLDEN, f"solve_{name}.npz"))
    a = synthetic(int(g["n"]), int(g["seed"]), electrons=int(g["electrons"]))
    s = v2g.V2RDMSolver.from_active_space(
        a, options=dict(R_CONVERGENCE=float(g["r_conv"]), E_CONVERGENCE=float(g["e_conv"])), start="feasible",
        projection="adaptive")
    e = s.compute_energy()
    assert s.result["status"] == 0
    assert abs(e - float(g["e_primal"])) <= 1e-6


# Options beyond the reference's loop (they change the path, not the answer); marked late,
# so that they run after every other test.


@pytest.mark.late
def test_cg_extrapolation_reaches_the_same_energy(v2g):
    # cg_extrapolate: CG starts from y_k + (y_k - y_{k-1}) with the reference's
    # stopping test, so the energy is the reference's and CG needs fewer
    # iterations.  Solved in one group with two instances that do not
    # extrapolate: the mode is per instance.
    from v2rdm_casscf_b200.hamiltonian import synthetic

    g = load(os.path.join(GOLDEN, "solve_synthetic_n4_s0.npz"))
    opts = dict(R_CONVERGENCE=float(g["r_conv"]), E_CONVERGENCE=float(g["e_conv"]))
    solvers = []
    for seed, ex in ((int(g["seed"]), True), (int(g["seed"]), False), (1, False)):
        s = v2g.V2RDMSolver.from_active_space(synthetic(4, seed), options=opts, cg_extrapolate=ex)
        s.guess()
        solvers.append(s)
    res = v2g.solve_batch(solvers)
    assert all(r["status"] == 0 for r in res)
    assert abs(res[0]["e_total"] - float(g["e_primal"])) <= 1e-6
    assert abs(res[1]["e_total"] - float(g["e_primal"])) <= 1e-6
    assert res[0]["iiter"] < res[1]["iiter"]
    g1 = load(os.path.join(GOLDEN, "solve_synthetic_n4_s1.npz"))
    assert abs(res[2]["e_total"] - float(g1["e_primal"])) <= 1e-6


@pytest.mark.late
def test_anderson_acceleration_reaches_the_same_energy(v2g):
    # anderson_memory: the stopping test and energies are the plain step's, so
    # the reference's energy is reached, in far fewer outer iterations.  One
    # group holds instances with memories 10, 5 and 0 (per-instance history
    # rings inside one allocation of 10 columns).
    from v2rdm_casscf_b200.hamiltonian import synthetic

    g = load(os.path.join(GOLDEN, "solve_synthetic_n4_s0.npz"))
    opts = dict(R_CONVERGENCE=float(g["r_conv"]), E_CONVERGENCE=float(g["e_conv"]))
    solvers = []
    for m in (10, 5, 0):
        s = v2g.V2RDMSolver.from_active_space(synthetic(4, int(g["seed"])), options=opts, anderson_memory=m,
                                              cg_extrapolate=m > 0)
        s.guess()
        solvers.append(s)
    res = v2g.solve_batch(solvers)
    assert all(r["status"] == 0 for r in res)
    for r in res:
        assert abs(r["e_total"] - float(g["e_primal"])) <= 1e-6
    assert res[0]["oiter"] <= 0.6 * res[2]["oiter"]
    assert res[1]["oiter"] <= 0.8 * res[2]["oiter"]


@pytest.mark.late
def test_tau_parameter_reaches_the_same_energy(v2g):
    # TAU_PARAMETER at the top of the plugin's documented range [1.0, 1.6]
    # (plugin.cc:94-97) changes the path, not the answer
    from v2rdm_casscf_b200.hamiltonian import synthetic

    g = load(os.path.join(GOLDEN, "solve_synthetic_n4_s0.npz"))
    s = v2g.V2RDMSolver.from_active_space(
        synthetic(4, int(g["seed"])),
        options=dict(R_CONVERGENCE=float(g["r_conv"]), E_CONVERGENCE=float(g["e_conv"]), TAU_PARAMETER=1.6),
        start="feasible")
    e = s.compute_energy()
    assert s.result["status"] == 0
    assert abs(e - float(g["e_primal"])) <= 1e-6


@pytest.mark.late
def test_cg_growth_stop_does_not_fire_in_converging_solves(v2g):
    # the CG safeguard against a right-hand side in the null space of A^T
    # (kCgGrowth, csrc/kernels.cuh) must never fire in a converging solve
    g, s = _solve_golden(v2g, "synthetic_n5_s2")
    e = s.compute_energy()
    assert s.result["status"] == 0 and s.result["cg_stalls"] == 0
    assert abs(e - float(g["e_primal"])) <= 1e-6


@pytest.mark.late
def test_segmented_solve_continues_the_loop(v2g):
    # one-step orbital optimisation runs the loop in segments with focas
    # between them (v2rdm_solver.cc:1855-1873): v2g_solve_continue carries
    # mu, the outer-iteration count (the mu schedule), eps(p) / eps(d) and
    # x, y, z across segments, so segments of 100 outer iterations with the
    # (here unchanged) integrals set again in between reach the reference's
    # energy in about the outer iterations of one solve
    from v2rdm_casscf_b200.hamiltonian import synthetic

    g = load(os.path.join(GOLDEN, "solve_synthetic_n4_s0.npz"))
    a = synthetic(4, int(g["seed"]))
    opts = dict(R_CONVERGENCE=float(g["r_conv"]), E_CONVERGENCE=float(g["e_conv"]))
    s1 = v2g.V2RDMSolver.from_active_space(a, options=opts)
    s1.guess()
    s1.compute_energy()
    s = v2g.V2RDMSolver.from_active_space(a, options=opts)
    s.guess()
    segments = 0
    while True:
        r = s.solve_continue(100)
        segments += 1
        if r["status"] == 0:
            break
        assert r["status"] == v2g.V2G_ERR_NOT_CONVERGED and segments < 100
        assert r["oiter"] == 100 * segments
        s.set_hamiltonian(a.oei_packed, a.qmo, a.nq, a.enuc)
    assert segments > 1
    assert abs(r["e_total"] - float(g["e_primal"])) <= 1e-6
    assert abs(r["oiter"] - s1.result["oiter"]) <= 0.05 * s1.result["oiter"]
