"""The reference arm of bench.py (the reference's CPU code, timed and
extrapolated) runs on the CPU and prints the contract's JSON line."""
import json
import os
import subprocess
import sys

from tests.helpers import ROOT


def _run(args):
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference"] + args,
                         capture_output=True, text=True, timeout=900, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    return json.loads(lines[0])


def test_reference_arm_prints_one_json_line(ref):
    d = _run(["--workload", "uniform8", "--count", "2", "--steps", "1", "--warmup", "0", "--cpu-sample", "8"])
    assert d["impl"] == "reference" and d["value"] > 0 and d["unit"] == "s"
    assert d["higher_is_better"] is False
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["cpu_baseline"]["kind"] == "reference"


def test_reference_arm_on_h10_uses_the_reference_counts(ref):
    # the default workload: the reference's time per CG iteration and per outer
    # iteration, sampled, times its own iteration counts for this input
    d = _run(["--steps", "1", "--warmup", "0"])
    assert d["impl"] == "reference" and d["config"]["workload"].startswith("h10")
    base = d["cpu_baseline"]
    assert base["extrapolated"] is True and "5371 outer" in base["sample"] and "152316 CG" in base["sample"]
    assert d["value"] == base["value"] > 0


def test_reference_counts_come_from_the_golden_solve():
    import bench

    oit, cgit, t, src = bench.reference_counts("h10")
    assert (oit, cgit) == (5371, 152316) and t > 0 and "solve_h10_chain" in src
    assert bench.reference_counts("batch256") is None
