"""Checkpoint and restart of the handle's state (the plugin's MU, PRIMAL,
DUAL 1, DUAL 2 entries); host code only, so it runs without a GPU."""
import numpy as np
import pytest


def test_checkpoint_round_trip(v2g, tmp_path):
    s = v2g.V2RDMSolver([5], 3, 2, 2)
    rng = np.random.default_rng(3)
    x, y, z = rng.standard_normal(s.dimx), rng.standard_normal(s.nconstraints), rng.standard_normal(s.dimx)
    s.set_state(x, y, z, 0.37)
    path = tmp_path / "v2rdm.ckpt"
    s.write_checkpoint(path)
    t = v2g.V2RDMSolver([5], 3, 2, 2)
    t.read_checkpoint(path)
    x2, y2, z2, mu2 = t.get_state()
    assert np.array_equal(x, x2) and np.array_equal(y, y2) and np.array_equal(z, z2) and mu2 == 0.37


def test_checkpoint_of_another_layout_is_refused(v2g, tmp_path):
    s = v2g.V2RDMSolver([4], 2, 2)
    s.guess()
    path = tmp_path / "a.ckpt"
    s.write_checkpoint(path)
    other = v2g.V2RDMSolver([5], 3, 2, 2)
    with pytest.raises(v2g.V2GError, match="different layout"):
        other.read_checkpoint(path)
    (tmp_path / "junk").write_bytes(b"not a checkpoint at all, just text")
    with pytest.raises(v2g.V2GError):
        s.read_checkpoint(tmp_path / "junk")
