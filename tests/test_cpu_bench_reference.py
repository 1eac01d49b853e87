"""The reference arm of bench.py (the reference's CPU code, timed and
extrapolated) runs on the CPU and prints the contract's JSON line."""
import json
import os
import subprocess
import sys

from tests.helpers import ROOT


def test_reference_arm_prints_one_json_line(ref):
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--workload",
                          "uniform8", "--count", "2", "--steps", "1", "--warmup", "0", "--cpu-sample", "8"],
                         capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["value"] > 0 and d["unit"] == "s"
    assert d["higher_is_better"] is False
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["cpu_baseline"]["kind"] == "reference"


def test_reference_iteration_counts_say_where_they_come_from():
    # the CPU baseline multiplies the reference's time per outer iteration by
    # an iteration count: the reference's own (recorded or golden) where there
    # is one, else this run's, flagged as an underestimate when the run's
    # start or loop options need fewer iterations than the reference's loop
    import types

    import bench

    def args(**kw):
        base = dict(workload="h50", count=1, start="state", anderson=0, cg_extrapolate=False, tau=1.0, mu_freq=500)
        base.update(kw)
        return types.SimpleNamespace(**base)

    counts, src = bench.reference_iterations(args(workload="h10", start="feasible", anderson=10), [1])
    assert counts == [5371] and "compiled reference" in src
    counts, src = bench.reference_iterations(args(), [123])
    assert counts == [123] and "the reference's loop and start" in src
    counts, src = bench.reference_iterations(args(anderson=10, cg_extrapolate=True, mu_freq=250), [123])
    assert counts == [123] and "underestimate" in src
