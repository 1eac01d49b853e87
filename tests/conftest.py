import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")
    config.addinivalue_line("markers", "late: runs after every other test (options beyond the reference's loop)")


def _has_gpu():
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    # tests of options beyond the reference's loop run after the parity tests,
    # so that a stop at the first failure (-x) never hides a parity result; the
    # allocation-free entry point's file (test_zz_*) stays the very last
    def rank(it):
        last = os.path.basename(str(it.fspath)).startswith("test_zz_")
        return (2 if last else (1 if "late" in it.keywords else 0))

    items[:] = sorted(items, key=rank)
    if _has_gpu():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def ref():
    """The compiled reference oracle (oracle/_ref); skips when it was not built."""
    from oracle import ref as R

    if not R.available():
        pytest.skip("oracle/_ref not built (make -C oracle)")
    return R


@pytest.fixture(scope="session")
def v2g():
    import v2rdm_casscf_b200 as V

    V.lib()  # raises if the library is missing: the product must be built
    return V
