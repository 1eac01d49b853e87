"""The product's constraint table against the reference's maps at the
benchmark's sizes, on the CPU: A exported from the product (v2g_export_A, the
operator the GPU kernels apply) times the seeded inputs of the map-checksum
fixtures, compared with the reference's bpsdp_Au / bpsdp_ATu outputs stored
there (sampled entries, largest magnitudes, projections); 1e-12 relative."""
import glob
import os
import sys

import numpy as np
import pytest

from tests.helpers import GOLDEN, csr_of, load

sys.path.insert(0, GOLDEN)


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "mapsum_*.npz"))),
                         ids=lambda p: os.path.basename(p))
def test_table_matches_reference_maps_at_size(v2g, path):
    from make_golden import mapsum_vectors

    g = load(path)
    n = int(g["n"])
    s = v2g.V2RDMSolver([n], n // 2, n // 2, options=dict(POSITIVITY=str(g["positivity"])))
    assert s.dimx == int(g["dimx"]) and s.nconstraints == int(g["ncon"])
    assert np.array_equal(s.dimensions, g["block_dims"])
    A = csr_of(s)
    u, w, pa, pt, ia, it = mapsum_vectors(s.dimx, s.nconstraints)
    au, atw = A @ u, A.T @ w
    assert np.abs(au[ia] - g["au"]).max() <= 1e-12 * float(g["au_max"])
    assert np.abs(atw[it] - g["atw"]).max() <= 1e-12 * float(g["atw_max"])
    assert abs(au @ pa - float(g["au_dot"])) <= 1e-12 * float(g["au_norm"]) * np.linalg.norm(pa)
    assert abs(atw @ pt - float(g["atw_dot"])) <= 1e-12 * float(g["atw_norm"]) * np.linalg.norm(pt)
