#!/usr/bin/env python3
"""Generates the golden fixtures in this directory from the reference itself.

Runs the reference's own hot-path code, compiled from the reference tree into
oracle/_ref/libv2rdm_ref.so (see oracle/Makefile), on seeded inputs and stores
inputs and outputs as .npz files:

  pack_<case>.npz   d1 and d2 of PackSpatialDensity for a seeded x
  maps_<case>.npz   A u and A^T w of bpsdp_Au / bpsdp_ATu for seeded u, w, plus
                    b (BuildConstraints) and the layout sizes
  c_<case>.npz      c and efzc of RepackIntegrals/FrozenCoreEnergy for seeded
                    integrals, with frozen/restricted orbitals
  xz_<case>.npz     Update_xz on a seeded state (x, y, z, mu) -> x, z
  solve_<case>.npz  a full BPSDP solve (random start, srand(0)) of a seeded
                    synthetic active space: final energies, iteration counts,
                    the per-iteration trace and the final x, y, z
  mapsum_<case>.npz A u and A^T w at sizes too large to store (n = 10 and 20
                    DQG, n = 6 and 8 DQGT2): seeded inputs, sampled outputs
                    and projections
  energy_<case>.npz a full BPSDP solve of an instance of the batched workload
                    (n = 8..20, seed = its index in the batch): energies,
                    iteration counts and CPU seconds only (the vectors of
                    these sizes are too large for a fixture)

Usage: python tests/golden/make_golden.py [part ...]   (needs `make -C oracle` first)
       parts: maps pack c xz solve h10 mapsum energy (default: all but mapsum
       and energy; energy takes about an hour of CPU time)
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle.ref import RefSolver, set_threads  # noqa: E402
from v2rdm_casscf_b200.hamiltonian import synthetic  # noqa: E402

MAP_CASES = {
    # name: (amopi, doccpi, soccpi, positivity, constrain_spin, constrain_sz)
    "c1_n4_dqg": ([4], [2], [0], "DQG", True, True),
    "c1_n6_dqg": ([6], [3], [0], "DQG", True, True),
    "c1_n5_triplet_dqg": ([5], [2], [1], "DQG", True, True),
    "c1_n5_dqg_nosz": ([5], [2], [1], "DQG", True, False),
    "c2v_dqg": ([2, 1, 1, 2], [1, 0, 0, 1], [0, 0, 0, 0], "DQG", True, True),
    "c1_n4_d": ([4], [2], [0], "D", True, True),
    "c1_n4_dqgt1": ([4], [2], [0], "DQGT1", True, True),
    "c1_n4_dqgt2": ([4], [2], [0], "DQGT2", True, True),
    "c2_n4_doublet_dqgt": ([2, 2], [1, 0], [1, 0], "DQGT1T2", True, True),
    # spin-adapted Q2 / G2 (SPIN_ADAPT_Q2, SPIN_ADAPT_G2); orbital energies in Pitzer order
    "c1_n4_dqg_saq2": ([4], [2], [0], "DQG", True, True, True, False),
    "c2v_dqg_saq2g2_nospin": ([2, 1, 1, 2], [1, 0, 0, 1], [0, 0, 0, 0], "DQG", False, True, True, True),
    # CONSTRAIN_D3
    "c1_n4_dqg_d3": ([4], [2], [0], "DQG", True, True, False, False, True),
    "c2_n5_doublet_d_d3": ([3, 2], [1, 1], [1, 0], "D", True, True, False, False, True),
    # CONSTRAIN_D4
    "c1_n4_dqg_d4": ([4], [2], [0], "DQG", True, True, False, False, True, True),
}

PACK_CASES = {
    # name: (amopi, doccpi, soccpi, orbital energies in Pitzer order or None)
    "c1_n4": ([4], [2], [0], None),
    "c1_n5_doublet": ([5], [2], [1], [0.5, 0.1, 0.3, 0.3, 0.2]),
    "c2v_n6": ([2, 1, 1, 2], [1, 0, 0, 1], [0, 0, 0, 0], [0.3, 1.1, 0.2, 0.5, 0.1, 0.9]),
    "c2_n5_doublet": ([3, 2], [1, 1], [1, 0], [0.2, 0.4, 0.9, 0.3, 0.35]),
}

# map checks at sizes whose vectors are too large for a fixture: the inputs are
# regenerated from the seed, and the fixture keeps 4096 sampled entries of A u
# and A^T w, their largest magnitudes and two projections onto seeded vectors
MAPSUM_CASES = {
    # name: (n, positivity)
    "c1_n10_dqg": (10, "DQG"),
    "c1_n20_dqg": (20, "DQG"),
    "c1_n6_dqgt2": (6, "DQGT2"),
    "c1_n8_dqgt2": (8, "DQGT2"),
}

# instances of the batched workload (bench.py batch256: n = batch_sizes(256)[seed]),
# solved by the reference to R_CONVERGENCE 1e-6 / E_CONVERGENCE 1e-7
ENERGY_CASES = {
    # name: (n, seed)
    "batch_n8_s3": (8, 3),
    "batch_n10_s40": (10, 40),
    "batch_n12_s13": (12, 13),
}

SOLVE_CASES = {
    # name: (n, seed, r_conv, e_conv, electrons[, positivity])
    "synthetic_n4_s0": (4, 0, 1e-6, 1e-7, None),
    "synthetic_n4_s1": (4, 1, 1e-6, 1e-7, None),
    "synthetic_n5_s2": (5, 2, 1e-6, 1e-7, None),      # singlet, N = 4
    "synthetic_n5_s2_doublet": (5, 2, 1e-6, 1e-7, 5),  # doublet, N = 5
    "synthetic_n4_s1_dqgt1": (4, 1, 1e-6, 1e-7, None, "DQGT1"),
    "synthetic_n4_s0_saq2": (4, 0, 1e-6, 1e-7, None, "DQG", True),   # SPIN_ADAPT_Q2
}


def maps(name, spec):
    amopi, docc, socc, pos, spin, sz = spec[:6]
    saq2, sag2 = (spec[6], spec[7]) if len(spec) > 6 else (False, False)
    d3 = spec[8] if len(spec) > 8 else False
    d4 = spec[9] if len(spec) > 9 else False
    extra = {}
    if saq2 or sag2:
        extra = dict(spin_adapt_q2=saq2, spin_adapt_g2=sag2, energies=np.arange(sum(amopi), dtype=float))
    if d3:
        extra["constrain_d3"] = True
    if d4:
        extra["constrain_d4"] = True
    r = RefSolver(amopi, docc, soccpi=socc, positivity=pos, constrain_spin=spin, constrain_sz=sz,
                  multiplicity=sum(socc) + 1, **extra)
    rng = np.random.default_rng(12345)
    u = rng.standard_normal(r.dimx)
    w = rng.standard_normal(r.ncon)
    r.build_constraints()
    np.savez_compressed(os.path.join(HERE, f"maps_{name}.npz"), amopi=amopi, doccpi=docc, soccpi=socc,
                        positivity=pos, constrain_spin=spin, constrain_sz=sz, dimx=r.dimx, ncon=r.ncon,
                        spin_adapt_q2=saq2, spin_adapt_g2=sag2, constrain_d3=d3, constrain_d4=d4,
                        block_dims=r.block_dims, u=u, w=w, Au=r.Au(u), ATw=r.ATu(w), b=r.get("b"))


def cvec():
    frzc, rstc, amo, rstv, frzv = [1, 0], [0, 1], [3, 2], [1, 0], [0, 1]
    docc, socc = [2, 2], [0, 0]
    nmopi = [frzc[h] + rstc[h] + amo[h] + rstv[h] + frzv[h] for h in range(2)]
    nfull = [nmopi[h] - frzv[h] for h in range(2)]
    nf = sum(nfull)
    rng = np.random.default_rng(7)
    oei = rng.standard_normal(sum(n * (n + 1) // 2 for n in nfull))
    nq = 7
    qmo = rng.standard_normal(nq * nf * (nf + 1) // 2)
    r = RefSolver(nmopi, docc, soccpi=socc, frzcpi=frzc, rstcpi=rstc, rstvpi=rstv, frzvpi=frzv)
    r.set_integrals(oei, qmo, nq)
    np.savez_compressed(os.path.join(HERE, "c_c2_core.npz"), frzc=frzc, rstc=rstc, amo=amo, rstv=rstv, frzv=frzv,
                        docc=docc, socc=socc, oei=oei, qmo=qmo, nq=nq, c=r.get("c"), efzc=r.efzc)


def xz():
    for n in (4, 6):
        r = RefSolver([n], [n // 2], positivity="DQG")
        a = synthetic(n, 3)
        r.set_integrals(a.oei_packed, a.qmo, a.nq)
        rng = np.random.default_rng(99 + n)
        x = rng.standard_normal(r.dimx)
        z = rng.standard_normal(r.dimx)
        y = rng.standard_normal(r.ncon)
        mu = 0.7
        r.set("x", x)
        r.set("y", y)
        r.set("z", z)
        r.update_xz(mu)
        np.savez_compressed(os.path.join(HERE, f"xz_n{n}.npz"), n=n, seed=3, x=x, y=y, z=z, mu=mu,
                            x_out=r.get("x"), z_out=r.get("z"))


def pack(name, spec):
    """PackSpatialDensity (v2rdm_solver.cc:3664-3773) of a seeded x."""
    amopi, docc, socc, energies = spec
    r = RefSolver(amopi, docc, soccpi=socc, multiplicity=sum(socc) + 1, energies=energies)
    x = np.random.default_rng(7).standard_normal(r.dimx)
    r.set("x", x)
    d1, d2 = r.pack_spatial_density()
    np.savez_compressed(os.path.join(HERE, f"pack_{name}.npz"), amopi=amopi, doccpi=docc, soccpi=socc,
                        energies=np.array(energies if energies is not None else [], dtype=float),
                        x=x, d1=d1, d2=d2)


def solve(name, spec):
    n, seed, rc, ec, electrons = spec[:5]
    pos = spec[5] if len(spec) > 5 else "DQG"
    saq2 = bool(spec[6]) if len(spec) > 6 else False
    a = synthetic(n, seed, electrons=electrons)
    r = RefSolver([n], [a.nb], soccpi=[a.na - a.nb], multiplicity=a.multiplicity, positivity=pos, spin_adapt_q2=saq2,
                  r_convergence=rc, e_convergence=ec)
    r.set_integrals(a.oei_packed, a.qmo, a.nq)
    r.guess()
    r.build_constraints()
    out = r.solve(trace_cap=100000)
    np.savez_compressed(os.path.join(HERE, f"solve_{name}.npz"), n=n, seed=seed, r_conv=rc, e_conv=ec,
                        electrons=a.na + a.nb, positivity=pos, spin_adapt_q2=saq2,
                        e_primal=out["e_primal"], e_dual=out["e_dual"], ep=out["ep"], ed=out["ed"],
                        oiter=out["oiter"], iiter=out["iiter"], converged=out["converged"], trace=out["trace"],
                        x=r.get("x"), y=r.get("y"), z=r.get("z"))


def mapsum_vectors(dimx, ncon, seed=2026):
    """The seeded inputs and projection vectors of a map-checksum fixture."""
    rng = np.random.default_rng(seed)
    u = rng.standard_normal(dimx)
    w = rng.standard_normal(ncon)
    pa = rng.standard_normal(ncon)
    pt = rng.standard_normal(dimx)
    ia = np.sort(rng.choice(ncon, size=min(4096, ncon), replace=False))
    it = np.sort(rng.choice(dimx, size=min(4096, dimx), replace=False))
    return u, w, pa, pt, ia, it


def mapsum(name, n, pos):
    r = RefSolver([n], [n // 2], positivity=pos)
    r.build_constraints()
    u, w, pa, pt, ia, it = mapsum_vectors(r.dimx, r.ncon)
    au, atw = r.Au(u), r.ATu(w)
    np.savez_compressed(os.path.join(HERE, f"mapsum_{name}.npz"), n=n, positivity=pos, dimx=r.dimx, ncon=r.ncon,
                        block_dims=r.block_dims, idx_a=ia, au=au[ia], idx_t=it, atw=atw[it],
                        au_max=np.abs(au).max(), atw_max=np.abs(atw).max(), au_dot=au @ pa, atw_dot=atw @ pt,
                        au_norm=np.linalg.norm(au), atw_norm=np.linalg.norm(atw))


def solve_energy(name, n, seed):
    """Reference solve of one batched-workload instance; energies and counts only."""
    from v2rdm_casscf_b200.hamiltonian import batch_sizes

    assert int(batch_sizes(256)[seed]) == n, "seed is not an n-orbital instance of the batch"
    a = synthetic(n, seed)
    r = RefSolver([n], [a.nb], soccpi=[a.na - a.nb], multiplicity=a.multiplicity, positivity="DQG",
                  r_convergence=1e-6, e_convergence=1e-7)
    r.set_integrals(a.oei_packed, a.qmo, a.nq)
    r.guess()
    r.build_constraints()
    out = r.solve()
    np.savez_compressed(os.path.join(HERE, f"energy_{name}.npz"), n=n, seed=seed, r_conv=1e-6, e_conv=1e-7,
                        electrons=a.na + a.nb, e_primal=out["e_primal"], e_dual=out["e_dual"], ep=out["ep"],
                        ed=out["ed"], oiter=out["oiter"], iiter=out["iiter"], converged=out["converged"],
                        t_total=out["t_total"], threads=int(os.environ.get("OMP_NUM_THREADS", "4")))


def solve_hchain(name, natoms, spacing):
    """Reference solve of an all-active H chain (STO-3G RHF orbitals, CD integrals)."""
    from v2rdm_casscf_b200.hchain import hydrogen_chain

    a = hydrogen_chain(natoms, spacing)
    n = a.n
    r = RefSolver([n], [a.nb], positivity="DQG", r_convergence=1e-6, e_convergence=1e-7)
    r.set_integrals(a.oei_packed, a.qmo, a.nq, a.enuc)
    r.guess()
    r.build_constraints()
    out = r.solve()
    np.savez_compressed(os.path.join(HERE, f"solve_{name}.npz"), n=n, natoms=natoms, spacing=spacing,
                        h=a.h, L=a.L, enuc=a.enuc, scf_energy=a.scf_energy, r_conv=1e-6, e_conv=1e-7,
                        e_primal=out["e_primal"], e_dual=out["e_dual"], ep=out["ep"], ed=out["ed"],
                        oiter=out["oiter"], iiter=out["iiter"], converged=out["converged"],
                        t_total=out["t_total"])


if __name__ == "__main__":
    set_threads(int(os.environ.get("OMP_NUM_THREADS", "4")))
    parts = sys.argv[1:] or ["maps", "pack", "c", "xz", "solve", "h10"]
    if "maps" in parts:
        for k, v in MAP_CASES.items():
            maps(k, v)
    if "pack" in parts:
        for k, v in PACK_CASES.items():
            pack(k, v)
    if "c" in parts:
        cvec()
    if "xz" in parts:
        xz()
    if "solve" in parts:
        for k, v in SOLVE_CASES.items():
            solve(k, v)
    if "h10" in parts:
        solve_hchain("h10_chain", 10, 0.9)
    if "mapsum" in parts:
        for k, v in MAPSUM_CASES.items():
            mapsum(k, *v)
    if "energy" in parts:
        for k, v in ENERGY_CASES.items():
            solve_energy(k, *v)
    print("golden fixtures written to", HERE)
