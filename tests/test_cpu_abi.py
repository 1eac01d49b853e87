"""The ctypes mirror of the C ABI has the layout of include/v2rdm_gpu.h:
every field of v2g_options, v2g_result and v2g_batch_stats at the offset the
C compiler gives it, and the same struct sizes.  A drift here would pass
wrong option values silently, so it is checked without a GPU by compiling a
probe against the header."""
import os
import subprocess
import tempfile

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _c_layout(struct, fields):
    src = ['#include <stdio.h>', '#include <stddef.h>', '#include "v2rdm_gpu.h"', "int main(void) {",
           f'  printf("%zu\\n", sizeof({struct}));']
    src += [f'  printf("%zu\\n", offsetof({struct}, {f}));' for f in fields]
    src += ["  return 0;", "}"]
    with tempfile.TemporaryDirectory() as d:
        c, exe = os.path.join(d, "probe.c"), os.path.join(d, "probe")
        with open(c, "w") as fh:
            fh.write("\n".join(src))
        subprocess.run(["gcc", "-std=c99", "-I", os.path.join(ROOT, "include"), c, "-o", exe], check=True)
        out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout.split()
    vals = [int(v) for v in out]
    return vals[0], vals[1:]


@pytest.mark.parametrize("cname,pyname", [("v2g_options", "Options"), ("v2g_result", "Result"),
                                          ("v2g_batch_stats", "BatchStats")])
def test_ctypes_struct_matches_header(cname, pyname):
    import ctypes

    import v2rdm_casscf_b200 as V

    cls = getattr(V, pyname)
    fields = [f[0] for f in cls._fields_]
    size, offsets = _c_layout(cname, fields)
    assert ctypes.sizeof(cls) == size
    assert [getattr(cls, f).offset for f in fields] == offsets


def test_solve_continue_checks_its_arguments():
    # v2g_solve_continue (one-step orbital optimisation segments): bad
    # arguments are refused before any device work; without a GPU the
    # solve reports V2G_ERR_NO_DEVICE instead of falling back to the CPU
    import ctypes

    import torch

    import v2rdm_casscf_b200 as V
    from v2rdm_casscf_b200.hamiltonian import synthetic

    L = V.lib()
    r = V.Result()
    assert L.v2g_solve_continue(None, 10, ctypes.byref(r)) == V.V2G_ERR_ARG
    s = V.V2RDMSolver.from_active_space(synthetic(4, 0))
    assert L.v2g_solve_continue(s.h, 0, ctypes.byref(r)) == V.V2G_ERR_ARG
    if not torch.cuda.is_available():
        assert L.v2g_solve_continue(s.h, 10, ctypes.byref(r)) == V.V2G_ERR_NO_DEVICE
