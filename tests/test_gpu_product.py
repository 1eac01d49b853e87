"""Parity at the benchmark's sizes and in the product's solve mode.

* Maps at n = 10 and n = 20 (DQG) and n = 6 and 8 (DQGT2) against the
  reference's bpsdp_Au / bpsdp_ATu: the fixtures keep sampled entries and
  projections of outputs too large to store (tests/golden/mapsum_*.npz), the
  inputs are regenerated from their seed.  1e-12 relative, as every map test.
* Instances of the batched workload (n = 8, 10, 12) solved by the reference
  to R_CONVERGENCE 1e-6 / E_CONVERGENCE 1e-7 (tests/golden/energy_*.npz):
  the GPU's plain FP64 solve and the product's mode must both land within
  1e-6 Eh of the reference's energy.
* The H10 chain in the product's mode (feasible start, adaptive and
  mixed-precision projection, Anderson acceleration, extrapolated CG start,
  MU_UPDATE_FREQUENCY 250): the benchmark's configuration, within 1e-6 Eh.
"""
import glob
import os
import sys

import numpy as np
import pytest

from tests.helpers import GOLDEN, load

pytestmark = pytest.mark.gpu

sys.path.insert(0, os.path.join(GOLDEN))

PRODUCT = dict(projection="adaptive", start="feasible", anderson_memory=10, cg_extrapolate=True,
               mixed_precision=True)


def _mapsum_vectors(dimx, ncon):
    from make_golden import mapsum_vectors

    return mapsum_vectors(dimx, ncon)


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "mapsum_*.npz"))),
                         ids=lambda p: os.path.basename(p))
def test_maps_match_reference_at_size(v2g, path):
    g = load(path)
    n = int(g["n"])
    s = v2g.V2RDMSolver([n], n // 2, n // 2, options=dict(POSITIVITY=str(g["positivity"])))
    assert s.dimx == int(g["dimx"]) and s.nconstraints == int(g["ncon"])
    u, w, pa, pt, ia, it = _mapsum_vectors(s.dimx, s.nconstraints)
    assert np.array_equal(ia, g["idx_a"]) and np.array_equal(it, g["idx_t"])
    au, atw = s.Au(u), s.ATu(w)
    assert abs(np.abs(au).max() - float(g["au_max"])) <= 1e-12 * float(g["au_max"])
    assert abs(np.abs(atw).max() - float(g["atw_max"])) <= 1e-12 * float(g["atw_max"])
    assert np.abs(au[ia] - g["au"]).max() <= 1e-12 * float(g["au_max"])
    assert np.abs(atw[it] - g["atw"]).max() <= 1e-12 * float(g["atw_max"])
    assert abs(au @ pa - float(g["au_dot"])) <= 1e-12 * float(g["au_norm"]) * np.linalg.norm(pa)
    assert abs(atw @ pt - float(g["atw_dot"])) <= 1e-12 * float(g["atw_norm"]) * np.linalg.norm(pt)


def _energy_cases():
    return sorted(glob.glob(os.path.join(GOLDEN, "energy_*.npz")))


@pytest.mark.parametrize("path", _energy_cases(), ids=lambda p: os.path.basename(p))
def test_batch_instances_match_reference(v2g, path):
    from v2rdm_casscf_b200.hamiltonian import synthetic

    g = load(path)
    a = synthetic(int(g["n"]), int(g["seed"]))
    opts = dict(R_CONVERGENCE=float(g["r_conv"]), E_CONVERGENCE=float(g["e_conv"]))
    plain = v2g.V2RDMSolver.from_active_space(a, options=opts)
    plain.guess()
    product = v2g.V2RDMSolver.from_active_space(a, options=dict(opts, MU_UPDATE_FREQUENCY=250), **PRODUCT)
    product.guess()
    res = v2g.solve_batch([plain]) + v2g.solve_batch([product])
    for r in res:
        assert r["status"] == 0
        assert abs(r["e_total"] - float(g["e_primal"])) <= 1e-6, (r["e_total"], float(g["e_primal"]))
    # the plain loop is the reference's: its iteration count is the reference's to a few percent
    assert abs(res[0]["oiter"] - int(g["oiter"])) <= 0.25 * int(g["oiter"])


def test_product_mode_h10_matches_reference(v2g):
    from v2rdm_casscf_b200.hamiltonian import ActiveSpace

    g = load(os.path.join(GOLDEN, "solve_h10_chain.npz"))
    a = ActiveSpace(g["h"], g["L"], 5, 5, enuc=float(g["enuc"]))
    s = v2g.V2RDMSolver.from_active_space(
        a, options=dict(R_CONVERGENCE=float(g["r_conv"]), E_CONVERGENCE=float(g["e_conv"]), MU_UPDATE_FREQUENCY=250),
        **PRODUCT)
    s.guess()
    e = s.compute_energy()
    assert s.result["status"] == 0
    assert abs(e - float(g["e_primal"])) <= 1e-6
    assert s.result["oiter"] < 0.5 * int(g["oiter"])


def test_mixed_precision_alone_reaches_the_same_energy(v2g):
    # only the mixed-precision projection on top of the reference's loop and start
    from v2rdm_casscf_b200.hamiltonian import ActiveSpace

    g = load(os.path.join(GOLDEN, "solve_h10_chain.npz"))
    a = ActiveSpace(g["h"], g["L"], 5, 5, enuc=float(g["enuc"]))
    s = v2g.V2RDMSolver.from_active_space(
        a, options=dict(R_CONVERGENCE=float(g["r_conv"]), E_CONVERGENCE=float(g["e_conv"])), projection="adaptive",
        mixed_precision=True)
    s.guess()
    e = s.compute_energy()
    assert s.result["status"] == 0
    assert abs(e - float(g["e_primal"])) <= 1e-6


@pytest.mark.late
def test_mixed_precision_on_tensor_cores_reaches_the_fp64_energy(v2g):
    # n = 16: the G2aa block of 512 takes the tensor-core phase (blocks padded to
    # 512 and more); the mixed solve must land on the FP64 solve's energy, whose
    # path is pinned to the reference's energies at n = 8..12 above
    from v2rdm_casscf_b200.hamiltonian import synthetic

    a = synthetic(16, 45)
    opts = dict(R_CONVERGENCE=1e-6, E_CONVERGENCE=1e-7, MU_UPDATE_FREQUENCY=250)
    kw = dict(PRODUCT)
    runs = []
    for mixed in (False, True):
        kw["mixed_precision"] = mixed
        s = v2g.V2RDMSolver.from_active_space(a, options=opts, **kw)
        s.guess()
        runs.append(v2g.solve_batch([s])[0])
    for r in runs:
        assert r["status"] == 0
    assert abs(runs[0]["e_total"] - runs[1]["e_total"]) <= 1e-6
